/*
 * internal.h -- private state of the CPU restatement oracle (test
 * infrastructure; see oracle.h).
 */
#ifndef FABIPB_ORACLE_INTERNAL_H
#define FABIPB_ORACLE_INTERNAL_H

#include <stddef.h>
#include "oracle.h"

#define OR_FOURPI_I (1.0 / (4.0 * 3.14159265358979323846))
#define OR_ONETHIRD 0.33333333333333333333333333

typedef struct {
  int n;          /* panels in tree order */
  double *vtx;    /* 9n */
  double *nrm;    /* 3n */
  double *area;   /* n */
  double *edge;   /* 9n: a[0]=v2-v1, a[1]=v0-v2, a[2]=v1-v0 (input.c:743-747) */
} or_panels;

/* one octree over points (panels via centroids, or charges) */
typedef struct {
  int depth, height;
  int nCubes;
  int *levStart;         /* cubes of level l: [levStart[l], levStart[l+1]) */
  int *level, *parent, *kidStart, *kidCount;
  int *itemStart, *itemCount;   /* contiguous range of (sorted) items */
  double *x, *rad, *lo, *up;    /* centre, eRad, box (levels >= height) */
  /* neighbour lists for levels >= height (getNbrs, gkSetup.c:363) */
  int *nbrStart, *nNbr1, *nNbr2, *nbr;
} or_tree;

struct or_sys {
  or_params p;
  double epsilon;        /* eps2/eps1 */
  int nIn;
  or_panels pn;          /* tree order */
  int *order;            /* tree index -> input index */
  or_tree t;
  /* expansion orders (gkSetup.c:42) */
  int maxOrder, *ordMom, *ordM2L, *nMom;
  /* index tables (expan.c:39-129) */
  int idxDim;            /* maxOrder + 3 */
  int *idx3;             /* idx3[(a*idxDim+b)*idxDim+c] */
  int *sgn3;
  double *fact, *ifact, *ifact3;
  /* flattened layouts (fmm.c:234-404) */
  int nLeaves, *leafStart, *leafCount;
  int nNear, *nearSrc, *nearDst, *nearOff;
  int nFmm, *fmmCube, *cubeFmm;
  int nM2L, *m2lSrc, *m2lDst;
  /* leaf Q2M/L2P matrices, column-major nMomLeaf x count per leaf */
  int nMomLeaf;
  double *Q2M0, *Q2M1;
  long long *leafMatOff;
  /* expansions per FMM cube, stride nMomMax */
  int nMomMax;
  double *momPot, *momDpdn, *lec1, *lec2, *lec3, *lec4;
  /* quadrature (numQuad.c:205-295) */
  double tLeg[11][10], wLeg[11][10];
  /* charges */
  int nChar;
  double *pos, *chr;
  int chargeTreeBuilt;
  or_tree ct;
  int *chgSorted;        /* charges in charge-tree leaf order */
  int *ctOrder;          /* per charge cube expansion order */
  double *ctMom;         /* per charge cube moments, stride nMomMax */
  /* preconditioner */
  int pcMode;
  int pcLevel, pcBlocks;
  int *pcStart, *pcSize;
  double **pcLU;
  int **pcPiv;
};

/* tree.c */
int or_build_tree(or_tree *t, int nItems, const double *pts, int depth, int height,
                  double minx, double miny, double minz, double length,
                  int *sortedItems);
void or_tree_boxes_panels(or_tree *t, const or_panels *pn);
void or_tree_boxes_points(or_tree *t, const double *pts, const int *sorted);
void or_tree_neighbours(or_tree *t, double eta0);
void or_tree_free(or_tree *t);

/* quad.c */
void or_init_quad(or_sys *s);
void or_kernel_ker4(double kappa, double eps, const double *x, const double *nX,
                    const double *nY, double *y);
void or_panel_ia0_raw(const or_sys *s, const or_panels *pn, int X, int Y, double out[4]);
void or_panel_rhs(const or_sys *s, int X, const double *chr, double out[2]);

/* expan.c */
void or_init_expan(or_sys *s);
void or_setup_derivs(const or_sys *s, int order, const double *x, double *d0, double *dk,
                     int coulombOnly);
void or_setup_fmm(or_sys *s);

/* threads */
typedef void (*or_range_fn)(void *ctx, int begin, int end);
void or_parallel_for(int n, int threads, or_range_fn fn, void *ctx);
int or_thread_count(const or_sys *s);

static inline int or_nmom(int p) { return ((p + 1) * (p + 2) * (p + 3)) / 6; }
static inline int or_idx3(const or_sys *s, int a, int b, int c) {
  return s->idx3[(a * s->idxDim + b) * s->idxDim + c];
}

#endif
