/*
 * tree.c -- restatement of the reference octree (test infrastructure).
 *
 * gkSetup.c builds a uniform-depth octree by walking each point down from the
 * root (goDown, gkSetup.c:142-183: child index ix+2iy+4iz from strict ">"
 * comparisons against minx+(i+0.5)*sideLen[level]), links cubes depth first
 * (linkcubes, :194-236: children in index order, empty ones dropped), takes
 * enclosing-box centres (getEnclBoxs, :264-322) and builds near/interaction
 * lists from the parent's near list (getNbrs, :363-437, MAC near(), :332-349).
 *
 * The depth-first order with children in index order is the order of the
 * Morton key whose 3-bit digit per level is (iz,iy,ix), so the restatement
 * computes that key with the same comparisons, stable-sorts the points by it
 * (points inside a leaf keep input order, as goDown appends them), and reads
 * every level's cubes off the sorted keys.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "internal.h"

typedef struct {
  unsigned long long key;
  int idx;
} keyidx;

static int cmp_keyidx(const void *a, const void *b) {
  const keyidx *x = (const keyidx *)a, *y = (const keyidx *)b;
  if (x->key < y->key) return -1;
  if (x->key > y->key) return 1;
  return (x->idx > y->idx) - (x->idx < y->idx);
}

int or_build_tree(or_tree *t, int n, const double *pts, int depth, int height,
                  double minx, double miny, double minz, double length,
                  int *sorted) {
  double sideLen[64];
  keyidx *ki = (keyidx *)malloc((size_t)n * sizeof(keyidx));
  int *cubeOf = (int *)malloc((size_t)n * sizeof(int));
  int *cubeOfPrev = (int *)malloc((size_t)n * sizeof(int));
  int lev, i, cap;

  memset(t, 0, sizeof(*t));
  if (depth < 1 || depth > 20 || n <= 0) { free(ki); free(cubeOf); free(cubeOfPrev); return 0; }
  t->depth = depth;
  t->height = height;
  for (lev = 0; lev <= depth; lev++) { sideLen[lev] = length; length *= 0.5; }

  for (i = 0; i < n; i++) {
    const double *x = &pts[3 * i];
    int ci = 0, cj = 0, ck = 0;
    unsigned long long key = 0ULL;
    for (lev = 0; lev < depth; lev++) {
      int ix = 0, iy = 0, iz = 0;
      if (x[0] > minx + (ci + 0.5) * sideLen[lev]) ix = 1;
      if (x[1] > miny + (cj + 0.5) * sideLen[lev]) iy = 1;
      if (x[2] > minz + (ck + 0.5) * sideLen[lev]) iz = 1;
      ci = 2 * ci + ix; cj = 2 * cj + iy; ck = 2 * ck + iz;
      key = (key << 3) | (unsigned long long)(ix + 2 * iy + 4 * iz);
    }
    ki[i].key = key;
    ki[i].idx = i;
  }
  qsort(ki, (size_t)n, sizeof(keyidx), cmp_keyidx);
  for (i = 0; i < n; i++) sorted[i] = ki[i].idx;

  cap = 16;
  t->levStart = (int *)calloc((size_t)depth + 2, sizeof(int));
  t->level = (int *)malloc((size_t)cap * sizeof(int));
  t->parent = (int *)malloc((size_t)cap * sizeof(int));
  t->itemStart = (int *)malloc((size_t)cap * sizeof(int));
  t->itemCount = (int *)malloc((size_t)cap * sizeof(int));
  t->nCubes = 0;
  for (lev = 0; lev <= depth; lev++) {
    int shift = 3 * (depth - lev);
    unsigned long long cur = 0ULL;
    t->levStart[lev] = t->nCubes;
    for (i = 0; i < n; i++) {
      unsigned long long pref = (shift >= 64) ? 0ULL : (ki[i].key >> shift);
      if (i == 0 || pref != cur) {
        if (t->nCubes == cap) {
          cap *= 2;
          t->level = (int *)realloc(t->level, (size_t)cap * sizeof(int));
          t->parent = (int *)realloc(t->parent, (size_t)cap * sizeof(int));
          t->itemStart = (int *)realloc(t->itemStart, (size_t)cap * sizeof(int));
          t->itemCount = (int *)realloc(t->itemCount, (size_t)cap * sizeof(int));
        }
        t->level[t->nCubes] = lev;
        t->parent[t->nCubes] = (lev == 0) ? -1 : cubeOfPrev[i];
        t->itemStart[t->nCubes] = i;
        t->itemCount[t->nCubes] = 0;
        t->nCubes++;
        cur = pref;
      }
      t->itemCount[t->nCubes - 1]++;
      cubeOf[i] = t->nCubes - 1;
    }
    memcpy(cubeOfPrev, cubeOf, (size_t)n * sizeof(int));
  }
  t->levStart[depth + 1] = t->nCubes;
  t->kidStart = (int *)malloc((size_t)t->nCubes * sizeof(int));
  t->kidCount = (int *)calloc((size_t)t->nCubes, sizeof(int));
  for (i = 0; i < t->nCubes; i++) t->kidStart[i] = -1;
  for (i = 0; i < t->nCubes; i++) {
    int p = t->parent[i];
    if (p >= 0) {
      if (t->kidStart[p] < 0) t->kidStart[p] = i;
      t->kidCount[p]++;
    }
  }
  t->x = (double *)calloc((size_t)t->nCubes * 3, sizeof(double));
  t->lo = (double *)calloc((size_t)t->nCubes * 3, sizeof(double));
  t->up = (double *)calloc((size_t)t->nCubes * 3, sizeof(double));
  t->rad = (double *)calloc((size_t)t->nCubes, sizeof(double));
  free(ki); free(cubeOf); free(cubeOfPrev);
  return 1;
}

static void finish_box(or_tree *t, int c) {
  double *lo = &t->lo[3 * c], *up = &t->up[3 * c];
  t->x[3 * c] = 0.5 * (lo[0] + up[0]);
  t->x[3 * c + 1] = 0.5 * (lo[1] + up[1]);
  t->x[3 * c + 2] = 0.5 * (lo[2] + up[2]);
  t->rad[c] = 0.5 * sqrt((up[0] - lo[0]) * (up[0] - lo[0]) + (up[1] - lo[1]) * (up[1] - lo[1]) +
                         (up[2] - lo[2]) * (up[2] - lo[2]));
}

static void parent_boxes(or_tree *t) {
  int lev, c, k, i;
  for (lev = t->depth - 1; lev >= t->height; lev--) {
    for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++) {
      double *lo = &t->lo[3 * c], *up = &t->up[3 * c];
      int k0 = t->kidStart[c];
      for (k = 0; k < 3; k++) { up[k] = t->up[3 * k0 + k]; lo[k] = t->lo[3 * k0 + k]; }
      for (i = 1; i < t->kidCount[c]; i++) {
        int kid = k0 + i;
        for (k = 0; k < 3; k++) {
          up[k] = t->up[3 * kid + k] > up[k] ? t->up[3 * kid + k] : up[k];
          lo[k] = t->lo[3 * kid + k] < lo[k] ? t->lo[3 * kid + k] : lo[k];
        }
      }
      finish_box(t, c);
    }
  }
}

/* getEnclBoxs, gkSetup.c:264-322: leaves from the panel vertices. */
void or_tree_boxes_panels(or_tree *t, const or_panels *pn) {
  int c, i, j, k;
  for (c = t->levStart[t->depth]; c < t->levStart[t->depth + 1]; c++) {
    double *lo = &t->lo[3 * c], *up = &t->up[3 * c];
    int p0 = t->itemStart[c];
    for (k = 0; k < 3; k++) { up[k] = pn->vtx[9 * p0 + k]; lo[k] = pn->vtx[9 * p0 + k]; }
    for (i = 0; i < t->itemCount[c]; i++) {
      int p = p0 + i;
      for (j = 0; j < 3; j++) {
        const double *x = &pn->vtx[9 * p + 3 * j];
        for (k = 0; k < 3; k++) {
          up[k] = x[k] > up[k] ? x[k] : up[k];
          lo[k] = x[k] < lo[k] ? x[k] : lo[k];
        }
      }
    }
    finish_box(t, c);
  }
  parent_boxes(t);
}

/* getChgEnclBoxs, chargeTree.c:178-222: leaves from the enclosed points. */
void or_tree_boxes_points(or_tree *t, const double *pts, const int *sorted) {
  int c, i, k;
  for (c = t->levStart[t->depth]; c < t->levStart[t->depth + 1]; c++) {
    double *lo = &t->lo[3 * c], *up = &t->up[3 * c];
    int s0 = t->itemStart[c];
    for (k = 0; k < 3; k++) { up[k] = lo[k] = pts[3 * sorted[s0] + k]; }
    for (i = 1; i < t->itemCount[c]; i++) {
      const double *x = &pts[3 * sorted[s0 + i]];
      for (k = 0; k < 3; k++) {
        up[k] = x[k] > up[k] ? x[k] : up[k];
        lo[k] = x[k] < lo[k] ? x[k] : lo[k];
      }
    }
    finish_box(t, c);
  }
  parent_boxes(t);
}

/* near(), gkSetup.c:332-349 */
static int or_near(const or_tree *t, int c1, int c2, double eta0) {
  double d0, d1, d2, dist, eta;
  if (c1 == c2) return 2;
  d0 = t->x[3 * c1] - t->x[3 * c2];
  d1 = t->x[3 * c1 + 1] - t->x[3 * c2 + 1];
  d2 = t->x[3 * c1 + 2] - t->x[3 * c2 + 2];
  dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (dist < 1e-15) return 1;
  eta = (t->rad[c1] + t->rad[c2]) / dist;
  return (eta < eta0) ? 0 : 1;
}

/* getNbrs, gkSetup.c:363-437 */
void or_tree_neighbours(or_tree *t, double eta0) {
  int nc = t->nCubes, lev, c;
  long long cap = 1024, used = 0;
  int *buf;
  t->nbrStart = (int *)malloc((size_t)nc * sizeof(int));
  t->nNbr1 = (int *)calloc((size_t)nc, sizeof(int));
  t->nNbr2 = (int *)calloc((size_t)nc, sizeof(int));
  t->nbr = (int *)malloc((size_t)cap * sizeof(int));
  for (c = 0; c < nc; c++) t->nbrStart[c] = -1;

  for (lev = t->height; lev <= t->depth; lev++) {
    for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++) {
      int cand = 0, nNbrs = 0, i1, i2, nP, nK, pos;
      /* candidate list: all level cubes at height, else parent-near kids */
      int *cands;
      if (lev == t->height) {
        cand = t->levStart[lev + 1] - t->levStart[lev];
        cands = (int *)malloc((size_t)cand * sizeof(int));
        for (pos = 0; pos < cand; pos++) cands[pos] = t->levStart[lev] + pos;
      } else {
        int p = t->parent[c];
        for (nP = 0; nP < t->nNbr1[p]; nP++) cand += t->kidCount[t->nbr[t->nbrStart[p] + nP]];
        cands = (int *)malloc((size_t)(cand > 0 ? cand : 1) * sizeof(int));
        pos = 0;
        for (nP = 0; nP < t->nNbr1[p]; nP++) {
          int np = t->nbr[t->nbrStart[p] + nP];
          for (nK = 0; nK < t->kidCount[np]; nK++) cands[pos++] = t->kidStart[np] + nK;
        }
      }
      for (pos = 0; pos < cand; pos++) if (or_near(t, c, cands[pos], eta0)) nNbrs++;
      while (used + cand > cap) {
        cap *= 2;
        t->nbr = (int *)realloc(t->nbr, (size_t)cap * sizeof(int));
      }
      buf = &t->nbr[used];
      t->nbrStart[c] = (int)used;
      for (pos = 0, i1 = 1, i2 = nNbrs; pos < cand; pos++) {
        int flag = or_near(t, c, cands[pos], eta0);
        if (flag == 1) buf[i1++] = cands[pos];
        else if (flag == 2) buf[0] = cands[pos];
        else buf[i2++] = cands[pos];
      }
      t->nNbr1[c] = i1;
      t->nNbr2[c] = i2;
      used += cand;
      free(cands);
    }
  }
}

void or_tree_free(or_tree *t) {
  free(t->levStart); free(t->level); free(t->parent); free(t->kidStart); free(t->kidCount);
  free(t->itemStart); free(t->itemCount); free(t->x); free(t->rad); free(t->lo); free(t->up);
  free(t->nbrStart); free(t->nNbr1); free(t->nNbr2); free(t->nbr);
  memset(t, 0, sizeof(*t));
}
