/*
 * core.c -- construction of the restatement oracle and the small accessors
 * (test infrastructure; see oracle.h).
 *
 *   panel edges a[0..2]                 input.c:743-747
 *   bounding cube + centroids           gkSetup.c:90-128 (loopPanels)
 *   expansion orders                    gkSetup.c:42-81 (getOrders)
 *   tree / boxes / neighbour lists      gkSetup.c:446-508 (gkInit), see tree.c
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include "internal.h"

int or_thread_count(const or_sys *s) {
  long hc = sysconf(_SC_NPROCESSORS_ONLN);
  int t = s->p.threads > 0 ? s->p.threads : (hc > 0 ? (int)hc : 1);
  return t < 1 ? 1 : (t > 128 ? 128 : t);
}

typedef struct {
  or_range_fn fn;
  void *ctx;
  int begin, end;
} par_task;

static void *par_worker(void *arg) {
  par_task *t = (par_task *)arg;
  t->fn(t->ctx, t->begin, t->end);
  return NULL;
}

void or_parallel_for(int n, int threads, or_range_fn fn, void *ctx) {
  pthread_t tid[128];
  par_task task[128];
  int t, created = 0;
  if (threads > n) threads = n;
  if (threads <= 1) { if (n > 0) fn(ctx, 0, n); return; }
  for (t = 0; t < threads; t++) {
    task[t].fn = fn; task[t].ctx = ctx;
    task[t].begin = (int)(((long long)n * t) / threads);
    task[t].end = (int)(((long long)n * (t + 1)) / threads);
  }
  for (t = 1; t < threads; t++) {
    if (pthread_create(&tid[t], NULL, par_worker, &task[t]) != 0) break;
    created++;
  }
  fn(ctx, task[0].begin, task[0].end);
  for (t = 1; t <= created; t++) pthread_join(tid[t], NULL);
  for (t = created + 1; t < threads; t++) fn(ctx, task[t].begin, task[t].end);
}

static void get_orders(or_sys *s) {
  int depth = s->p.depth, height = s->p.height, order = s->p.order, lev;
  s->ordMom = (int *)calloc((size_t)depth + 1, sizeof(int));
  s->ordM2L = (int *)calloc((size_t)depth + 1, sizeof(int));
  if (order > 0) {
    for (lev = 0; lev <= depth; lev++) { s->ordM2L[lev] = order; s->ordMom[lev] = order; }
    s->maxOrder = order;
  } else {
    s->ordM2L[depth] = -order;
    for (lev = depth - 1; lev >= height; lev--) s->ordM2L[lev] = s->ordM2L[lev + 1] + 1;
    s->maxOrder = s->ordM2L[height];
    for (lev = depth; lev >= height; lev--) {
      if (s->p.order_mom >= 0) {
        int o = s->ordM2L[lev] + s->p.order_mom;
        s->ordMom[lev] = o < s->maxOrder ? o : s->maxOrder;
      } else {
        s->ordMom[lev] = s->maxOrder;
      }
    }
  }
  s->nMom = (int *)calloc((size_t)s->maxOrder + 3, sizeof(int));
  for (lev = 0; lev <= s->maxOrder + 2; lev++) s->nMom[lev] = or_nmom(lev);
}

or_sys *or_create(const or_params *prm, int n, const double *vtx, const double *normal,
                  const double *area) {
  or_sys *s = (or_sys *)calloc(1, sizeof(or_sys));
  double minx, miny, minz, maxx, maxy, maxz, length;
  double *ctr;
  int i, k, j;
  s->p = *prm;
  s->epsilon = prm->eps2 / prm->eps1;
  s->nIn = n;
  or_init_quad(s);
  /* loopPanels: extents over every vertex, centroid ONETHIRD*(v0+v1+v2) */
  minx = maxx = vtx[0]; miny = maxy = vtx[1]; minz = maxz = vtx[2];
  ctr = (double *)malloc((size_t)n * 3 * sizeof(double));
  for (i = 0; i < n; i++) {
    const double *v = &vtx[9 * i];
    for (k = 0; k < 3; k++) {
      const double *x = &v[3 * k];
      maxx = x[0] > maxx ? x[0] : maxx; minx = minx > x[0] ? x[0] : minx;
      maxy = x[1] > maxy ? x[1] : maxy; miny = miny > x[1] ? x[1] : miny;
      maxz = x[2] > maxz ? x[2] : maxz; minz = minz > x[2] ? x[2] : minz;
    }
    for (k = 0; k < 3; k++) ctr[3 * i + k] = OR_ONETHIRD * (v[k] + v[3 + k] + v[6 + k]);
  }
  length = (maxx - minx) > (maxy - miny) ? (maxx - minx) : (maxy - miny);
  length = (maxz - minz) > length ? (maxz - minz) : length;
  s->order = (int *)malloc((size_t)n * sizeof(int));
  if (!or_build_tree(&s->t, n, ctr, prm->depth, prm->height, minx, miny, minz, length, s->order)) {
    free(ctr); free(s);
    return NULL;
  }
  free(ctr);
  /* panels permuted to tree order */
  s->pn.n = n;
  s->pn.vtx = (double *)malloc((size_t)n * 9 * sizeof(double));
  s->pn.nrm = (double *)malloc((size_t)n * 3 * sizeof(double));
  s->pn.area = (double *)malloc((size_t)n * sizeof(double));
  s->pn.edge = (double *)malloc((size_t)n * 9 * sizeof(double));
  for (i = 0; i < n; i++) {
    int o = s->order[i];
    double *v = &s->pn.vtx[9 * i], *e = &s->pn.edge[9 * i];
    memcpy(v, &vtx[9 * o], 9 * sizeof(double));
    memcpy(&s->pn.nrm[3 * i], &normal[3 * o], 3 * sizeof(double));
    s->pn.area[i] = area[o];
    for (j = 0; j < 3; j++) {
      e[j] = v[6 + j] - v[3 + j];       /* a[0] = v2 - v1 */
      e[3 + j] = v[j] - v[6 + j];       /* a[1] = v0 - v2 */
      e[6 + j] = v[3 + j] - v[j];       /* a[2] = v1 - v0 */
    }
  }
  or_tree_boxes_panels(&s->t, &s->pn);
  or_tree_neighbours(&s->t, prm->sep_ratio);
  get_orders(s);
  or_init_expan(s);
  or_setup_fmm(s);
  return s;
}

int or_num_panels(const or_sys *s) { return s->pn.n; }
int or_num_leaves(const or_sys *s) { return s->nLeaves; }
int or_num_near_pairs(const or_sys *s) { return s->nNear; }
int or_num_m2l_pairs(const or_sys *s) { return s->nM2L; }
int or_num_cubes(const or_sys *s) { return s->nFmm; }
int or_max_order(const or_sys *s) { return s->maxOrder; }

void or_panel_order(const or_sys *s, int *order) { memcpy(order, s->order, (size_t)s->pn.n * sizeof(int)); }

void or_leaf_layout(const or_sys *s, int *start, int *count) {
  memcpy(start, s->leafStart, (size_t)s->nLeaves * sizeof(int));
  memcpy(count, s->leafCount, (size_t)s->nLeaves * sizeof(int));
}

void or_near_pairs(const or_sys *s, int *src, int *dst) {
  memcpy(src, s->nearSrc, (size_t)s->nNear * sizeof(int));
  memcpy(dst, s->nearDst, (size_t)s->nNear * sizeof(int));
}

void or_m2l_pairs(const or_sys *s, int *src, int *dst) {
  memcpy(src, s->m2lSrc, (size_t)s->nM2L * sizeof(int));
  memcpy(dst, s->m2lDst, (size_t)s->nM2L * sizeof(int));
}

void or_cube_data(const or_sys *s, int *level, int *count, double *ctr4) {
  int f;
  for (f = 0; f < s->nFmm; f++) {
    int c = s->fmmCube[f];
    level[f] = s->t.level[c];
    count[f] = s->t.itemCount[c];
    ctr4[4 * f] = s->t.x[3 * c];
    ctr4[4 * f + 1] = s->t.x[3 * c + 1];
    ctr4[4 * f + 2] = s->t.x[3 * c + 2];
    ctr4[4 * f + 3] = s->t.rad[c];
  }
}

void or_area_tree(const or_sys *s, double *area) { memcpy(area, s->pn.area, (size_t)s->pn.n * sizeof(double)); }

void or_panel_ia0(const or_sys *s, int x, int y, double out[4]) { or_panel_ia0_raw(s, &s->pn, x, y, out); }

void or_destroy(or_sys *s) {
  int b;
  if (s == NULL) return;
  or_tree_free(&s->t);
  or_tree_free(&s->ct);
  free(s->order); free(s->pn.vtx); free(s->pn.nrm); free(s->pn.area); free(s->pn.edge);
  free(s->ordMom); free(s->ordM2L); free(s->nMom); free(s->idx3); free(s->sgn3);
  free(s->fact); free(s->ifact); free(s->ifact3);
  free(s->leafStart); free(s->leafCount); free(s->nearSrc); free(s->nearDst); free(s->nearOff);
  free(s->fmmCube); free(s->cubeFmm); free(s->m2lSrc); free(s->m2lDst);
  free(s->Q2M0); free(s->Q2M1); free(s->leafMatOff);
  free(s->momPot); free(s->momDpdn); free(s->lec1); free(s->lec2); free(s->lec3); free(s->lec4);
  free(s->pos); free(s->chr); free(s->chgSorted); free(s->ctOrder); free(s->ctMom);
  for (b = 0; b < s->pcBlocks; b++) { if (s->pcLU) free(s->pcLU[b]); if (s->pcPiv) free(s->pcPiv[b]); }
  free(s->pcLU); free(s->pcPiv); free(s->pcStart); free(s->pcSize);
  free(s);
}
