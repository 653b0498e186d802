/*
 * oracle.h -- CPU restatement of the FABIPB hot path.  TEST INFRASTRUCTURE:
 * only the tests, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
 * call this, and only as the checker; the product never links it.
 *
 * Everything is FP64 and follows the reference's arithmetic and loop order
 * (file:line citations on each function), so that on the same panels the
 * results agree with the reference binary to rounding.  Parity of this file
 * with the reference is pinned by tests/test_oracle_pin.py, which runs the
 * reference compiled from its own sources (oracle/_ref/) on the same inputs.
 *
 * Arrays are flat and in the reference's conventions:
 *   panels in input order: vtx[9*i + 3*k + d] = vertex k, coordinate d
 *   vectors of unknowns: x[0..N) potential part, x[N..2N) normal-derivative
 *   part, both in tree (pnlLst) order.
 */
#ifndef FABIPB_ORACLE_H
#define FABIPB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_params {
  int order;          /* -p : >0 fixed order, <=0 variable order (gkSetup.c:42) */
  int order_mom;      /* -pm */
  int depth;          /* -t */
  int height;         /* -H */
  int quad_order;     /* -q */
  double sep_ratio;   /* -S */
  double kappa;       /* -k */
  double eps1, eps2;  /* -eps1 -eps2 */
  double rhs_theta;   /* FABIPB_RHS_TREE_THETA (default 0.8) */
  double energy_theta;/* FABIPB_ENERGY_TREE_THETA (default 0.8) */
  int charge_order;   /* charge-tree order: >0 flat, 0 follow the FMM (chargeTree.c:117) */
  int threads;        /* worker threads for the heavy loops (<=0: all online CPUs) */
} or_params;

typedef struct or_sys or_sys;

or_sys *or_create(const or_params *prm, int n, const double *vtx,
                  const double *normal, const double *area);
void or_destroy(or_sys *s);
int or_set_charges(or_sys *s, int m, const double *pos, const double *q);

/* tree queries (after or_create) */
int or_num_panels(const or_sys *s);
int or_num_leaves(const or_sys *s);
int or_num_near_pairs(const or_sys *s);
int or_num_m2l_pairs(const or_sys *s);
int or_num_cubes(const or_sys *s);
int or_max_order(const or_sys *s);
void or_panel_order(const or_sys *s, int *order);          /* tree index -> input index */
void or_leaf_layout(const or_sys *s, int *start, int *count);
void or_near_pairs(const or_sys *s, int *src, int *dst);    /* reference buildApplyLayout order */
void or_m2l_pairs(const or_sys *s, int *src, int *dst);     /* reference buildM2LPairList order */
void or_cube_data(const or_sys *s, int *level, int *count, double *ctr4);
void or_area_tree(const or_sys *s, double *area);

/* one panel pair, the Galerkin coefficient of panelIA0 (numQuad.c:629) */
void or_panel_ia0(const or_sys *s, int x_tree, int y_tree, double out[4]);

/* operators, in tree order */
void or_near_apply(or_sys *s, double alpha, const double *sgm, double *pot);
void or_fmm_apply(or_sys *s, double alpha, const double *sgm, double beta, double *pot);
void or_matvec(or_sys *s, double alpha, const double *x, double beta, double *y);
void or_far_apply(or_sys *s, double alpha, const double *sgm, double beta, double *pot);

/* right-hand side and energy */
void or_rhs_direct(or_sys *s, double *rhs);
void or_rhs_tree(or_sys *s, double *rhs);
double or_energy_tree(or_sys *s, const double *sgm);   /* raw sum, before 2*pi*332.0716 */

/* preconditioner and solve */
int or_precond_setup(or_sys *s, int mode);   /* 2 = cached block LU, 3 = diagonal, -1 none */
void or_precond_apply(or_sys *s, const double *b, double *x);
int or_gmres(or_sys *s, const double *b, double *x, int restart, int *iter,
             double *resid);

#ifdef __cplusplus
}
#endif
#endif
