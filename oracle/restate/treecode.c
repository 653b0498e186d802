/*
 * treecode.c -- restatement of the charge tree, the right-hand side and the
 * post-solve energy (test infrastructure).
 *
 *   charge octree + boxes              chargeTree.c:136-307 (buildChargeTree)
 *   charge-tree expansion order         chargeTree.c:117-129
 *   leaf / upward charge moments        chargeTree.c:314-416
 *   direct RHS                          fabipb.c:788-798 + numQuad.c:786-819
 *   tree RHS walk                       treecode.c:283-450 (rhsTreeWalkLocal)
 *   panel-tree energy walk              treecode.c:581-695, 869-887
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "internal.h"

int or_set_charges(or_sys *s, int m, const double *pos, const double *q) {
  free(s->pos); free(s->chr);
  s->nChar = m;
  s->pos = (double *)malloc((size_t)m * 3 * sizeof(double));
  s->chr = (double *)malloc((size_t)m * sizeof(double));
  memcpy(s->pos, pos, (size_t)m * 3 * sizeof(double));
  memcpy(s->chr, q, (size_t)m * sizeof(double));
  if (s->chargeTreeBuilt) {
    or_tree_free(&s->ct);
    free(s->chgSorted); free(s->ctOrder); free(s->ctMom);
    s->chgSorted = NULL; s->ctOrder = NULL; s->ctMom = NULL;
    s->chargeTreeBuilt = 0;
  }
  return 1;
}

static int charge_order(const or_sys *s, int level) {
  int order;
  if (s->p.charge_order > 0) order = s->p.charge_order;
  else order = s->ordMom[level] > 4 ? s->ordMom[level] : 4;
  return order < s->maxOrder ? order : s->maxOrder;
}

static void build_charge_tree(or_sys *s) {
  int m = s->nChar, j, lev, c, i, k;
  double cminx, cmaxx, cminy, cmaxy, cminz, cmaxz, length;
  or_tree *t = &s->ct;
  size_t M = (size_t)s->nMomMax;
  if (s->chargeTreeBuilt) return;
  cminx = cmaxx = s->pos[0]; cminy = cmaxy = s->pos[1]; cminz = cmaxz = s->pos[2];
  for (j = 1; j < m; j++) {
    double x = s->pos[3 * j], y = s->pos[3 * j + 1], z = s->pos[3 * j + 2];
    cminx = cminx > x ? x : cminx; cmaxx = x > cmaxx ? x : cmaxx;
    cminy = cminy > y ? y : cminy; cmaxy = y > cmaxy ? y : cmaxy;
    cminz = cminz > z ? z : cminz; cmaxz = z > cmaxz ? z : cmaxz;
  }
  length = (cmaxx - cminx) > (cmaxy - cminy) ? (cmaxx - cminx) : (cmaxy - cminy);
  length = (cmaxz - cminz) > length ? (cmaxz - cminz) : length;
  if (length <= 0.0) length = 1.0;
  s->chgSorted = (int *)malloc((size_t)m * sizeof(int));
  or_build_tree(t, m, s->pos, s->t.depth, s->t.height, cminx, cminy, cminz, length, s->chgSorted);
  or_tree_boxes_points(t, s->pos, s->chgSorted);
  /* moments: leaves directly, parents by M2M (computeChgMoments) */
  s->ctOrder = (int *)calloc((size_t)t->nCubes, sizeof(int));
  s->ctMom = (double *)calloc((size_t)t->nCubes * M, sizeof(double));
  for (c = 0; c < t->nCubes; c++) s->ctOrder[c] = (t->level[c] >= t->height) ? charge_order(s, t->level[c]) : 0;
  {
    double cv[512], f1[64], f2[64], f3[64];
    for (c = t->levStart[t->depth]; c < t->levStart[t->depth + 1]; c++) {
      int order = s->ctOrder[c], nMom = or_nmom(order);
      double *mom = &s->ctMom[c * M];
      for (k = 0; k < t->itemCount[c]; k++) {
        int jj = s->chgSorted[t->itemStart[c] + k], n, i1, i2;
        double trns[3];
        trns[0] = s->pos[3 * jj] - t->x[3 * c];
        trns[1] = s->pos[3 * jj + 1] - t->x[3 * c + 1];
        trns[2] = s->pos[3 * jj + 2] - t->x[3 * c + 2];
        f1[0] = f2[0] = f3[0] = 1.0;
        for (i = 1; i <= order; i++) {
          f1[i] = f1[i - 1] * trns[0]; f2[i] = f2[i - 1] * trns[1]; f3[i] = f3[i - 1] * trns[2];
        }
        for (i = n = 0; n <= order; n++)
          for (i1 = 0; i1 <= n; i1++)
            for (i2 = 0; i2 <= n - i1; i2++, i++) {
              cv[i] = f1[i1] * f2[i2] * f3[n - i1 - i2];
              cv[i] *= s->ifact3[i];
            }
        for (i = 0; i < nMom; i++) mom[i] += s->chr[jj] * cv[i];
      }
    }
    for (lev = t->depth - 1; lev >= t->height; lev--) {
      for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++) {
        int ordOut = s->ctOrder[c];
        for (k = 0; k < t->kidCount[c]; k++) {
          int kid = t->kidStart[c] + k, ordIn = s->ctOrder[kid], nIn = or_nmom(ordIn);
          int n, i1, i2, i3, k1, k2, k3;
          double trns[3];
          for (i = 0; i < 3; i++) trns[i] = t->x[3 * kid + i] - t->x[3 * c + i];
          f1[0] = f2[0] = f3[0] = 1.0;
          for (i = 1; i <= ordOut; i++) {
            f1[i] = f1[i - 1] * trns[0]; f2[i] = f2[i - 1] * trns[1]; f3[i] = f3[i - 1] * trns[2];
          }
          for (i = n = 0; n <= ordOut; n++)
            for (i1 = 0; i1 <= n; i1++)
              for (i2 = 0; i2 <= n - i1; i2++, i++) {
                cv[i] = f1[i1] * f2[i2] * f3[n - i1 - i2];
                cv[i] *= s->ifact3[i];
              }
          for (i = n = 0; n <= ordOut; n++)
            for (i1 = 0; i1 <= n; i1++)
              for (i2 = 0; i2 <= n - i1; i2++, i++) {
                double tmp = 0.0;
                i3 = n - i1 - i2;
                for (k1 = 0; k1 <= i1; k1++)
                  for (k2 = 0; k2 <= i2; k2++)
                    for (k3 = 0; k3 <= i3; k3++) {
                      int b = or_idx3(s, k1, k2, k3);
                      if (b < nIn) tmp += cv[or_idx3(s, i1 - k1, i2 - k2, i3 - k3)] * s->ctMom[kid * M + b];
                    }
                s->ctMom[c * M + i] += tmp;
              }
        }
      }
    }
  }
  s->chargeTreeBuilt = 1;
}

/* one charge-tree walk at a target point (mode 0 RHS, mode 1 energy) */
static void tree_walk(or_sys *s, int c, const double *qp, const double *nrm, int mode,
                      double *d0, double *dk, double *y) {
  const or_tree *t = &s->ct;
  double r[3], dist, theta = (mode == 0) ? s->p.rhs_theta : s->p.energy_theta;
  int k, i;
  for (k = 0; k < 3; k++) r[k] = qp[k] - t->x[3 * c + k];
  dist = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  if (t->rad[c] < theta * dist && t->level[c] >= s->t.height) {
    int order = s->ctOrder[c], n, i1, i2, i3;
    const double *mom = &s->ctMom[(size_t)c * s->nMomMax];
    double y0 = 0.0, y1 = 0.0;
    or_setup_derivs(s, order + 1, r, d0, dk, mode == 0);
    for (i = n = 0; n <= order; n++)
      for (i1 = 0; i1 <= n; i1++)
        for (i2 = 0; i2 <= n - i1; i2++, i++) {
          i3 = n - i1 - i2;
          if (mode == 0) {
            double dn;
            y0 += s->sgn3[i] * mom[i] * d0[i];
            dn = nrm[0] * d0[or_idx3(s, i1 + 1, i2, i3)] + nrm[1] * d0[or_idx3(s, i1, i2 + 1, i3)] +
                 nrm[2] * d0[or_idx3(s, i1, i2, i3 + 1)];
            y1 += s->sgn3[i] * mom[i] * dn;
          } else {
            double dn0, dnk;
            y0 += s->sgn3[i] * mom[i] * (d0[i] - dk[i]);
            dn0 = nrm[0] * d0[or_idx3(s, i1 + 1, i2, i3)] + nrm[1] * d0[or_idx3(s, i1, i2 + 1, i3)] +
                  nrm[2] * d0[or_idx3(s, i1, i2, i3 + 1)];
            dnk = nrm[0] * dk[or_idx3(s, i1 + 1, i2, i3)] + nrm[1] * dk[or_idx3(s, i1, i2 + 1, i3)] +
                  nrm[2] * dk[or_idx3(s, i1, i2, i3 + 1)];
            y1 += s->sgn3[i] * mom[i] * (s->epsilon * dnk - dn0);
          }
        }
    if (mode == 0) { y[0] += y0 / OR_FOURPI_I; y[1] += y1 / OR_FOURPI_I; }
    else { y[0] += y0; y[1] += y1; }
    return;
  }
  if (t->level[c] == t->depth) {
    for (i = 0; i < t->itemCount[c]; i++) {
      int j = s->chgSorted[t->itemStart[c] + i];
      double x[3], r2;
      for (k = 0; k < 3; k++) x[k] = qp[k] - s->pos[3 * j + k];
      r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
      if (mode == 0) {
        double ri = 1.0 / sqrt(r2), r3i = ri / r2;
        double ip = nrm[0] * x[0] + nrm[1] * x[1] + nrm[2] * x[2];
        y[0] += s->chr[j] * ri;
        y[1] += s->chr[j] * (-ip * r3i);
      } else {
        double rn = sqrt(r2), G0 = OR_FOURPI_I / rn;
        double Gk = exp(-s->p.kappa * rn) * G0;
        double coef = (s->p.kappa * rn + 1.0) * exp(-s->p.kappa * rn);
        double ip = nrm[0] * x[0] + nrm[1] * x[1] + nrm[2] * x[2];
        double dG0dn = -ip * G0 / r2, dGkdn = coef * dG0dn;
        y[0] += s->chr[j] * (G0 - Gk);
        y[1] += s->chr[j] * (s->epsilon * dGkdn - dG0dn);
      }
    }
    return;
  }
  for (i = 0; i < t->kidCount[c]; i++) tree_walk(s, t->kidStart[c] + i, qp, nrm, mode, d0, dk, y);
}

typedef struct {
  or_sys *s;
  int mode;
  const double *sgm;
  double *out;        /* mode 0: rhs (2N); mode 1: per-panel energy terms (N) */
} walk_ctx;

static void walk_range(void *vctx, int begin, int end) {
  walk_ctx *w = (walk_ctx *)vctx;
  or_sys *s = w->s;
  int q = s->p.quad_order, n = s->pn.n, X, ix, jx, k;
  size_t nd = (size_t)or_nmom(s->maxOrder + 2);
  double *d0 = (double *)malloc(nd * sizeof(double)), *dk = (double *)malloc(nd * sizeof(double));
  double fac = OR_FOURPI_I / s->p.eps1;
  for (X = begin; X < end; X++) {
    const double *v0 = &s->pn.vtx[9 * X], *ax2 = &s->pn.edge[9 * X + 6], *ax0 = &s->pn.edge[9 * X];
    const double *nrm = &s->pn.nrm[3 * X];
    const double *t = s->tLeg[q], *wl = s->wLeg[q];
    double out0 = 0.0, out1 = 0.0;
    for (ix = 0; ix < q; ix++)
      for (jx = 0; jx < q; jx++) {
        double r[3], y[2] = {0.0, 0.0};
        for (k = 0; k < 3; k++) r[k] = v0[k] + t[ix] * (ax2[k] + t[jx] * ax0[k]);
        tree_walk(s, 0, r, nrm, w->mode, d0, dk, y);
        out0 += y[0] * t[ix] * wl[ix] * wl[jx];
        out1 += y[1] * t[ix] * wl[ix] * wl[jx];
      }
    out0 *= 2.0 * s->pn.area[X];
    out1 *= 2.0 * s->pn.area[X];
    if (w->mode == 0) {
      w->out[X] = fac * out0;
      w->out[n + X] = fac * out1;
    } else {
      w->out[X] = out0 * w->sgm[X + n] + out1 * w->sgm[X];
    }
  }
  free(d0); free(dk);
}

void or_rhs_tree(or_sys *s, double *rhs) {
  walk_ctx w;
  build_charge_tree(s);
  w.s = s; w.mode = 0; w.sgm = NULL; w.out = rhs;
  or_parallel_for(s->pn.n, or_thread_count(s), walk_range, &w);
}

double or_energy_tree(or_sys *s, const double *sgm) {
  walk_ctx w;
  double e = 0.0;
  int i;
  build_charge_tree(s);
  w.s = s; w.mode = 1; w.sgm = sgm; w.out = (double *)malloc((size_t)s->pn.n * sizeof(double));
  or_parallel_for(s->pn.n, or_thread_count(s), walk_range, &w);
  for (i = 0; i < s->pn.n; i++) e += w.out[i];
  free(w.out);
  return e;
}

typedef struct {
  or_sys *s;
  double *rhs;
} rhs_ctx;

static void rhs_direct_range(void *vctx, int begin, int end) {
  rhs_ctx *c = (rhs_ctx *)vctx;
  or_sys *s = c->s;
  int n = s->pn.n, i, j;
  double fac = OR_FOURPI_I / s->p.eps1;
  for (i = begin; i < end; i++) {
    double a = 0.0, b = 0.0;
    for (j = 0; j < s->nChar; j++) {
      double out[2];
      or_panel_rhs(s, i, &s->pos[3 * j], out);
      a += s->chr[j] * out[0];
      b += s->chr[j] * out[1];
    }
    c->rhs[i] = a * fac;
    c->rhs[n + i] = b * fac;
  }
}

void or_rhs_direct(or_sys *s, double *rhs) {
  rhs_ctx c;
  c.s = s; c.rhs = rhs;
  or_parallel_for(s->pn.n, or_thread_count(s), rhs_direct_range, &c);
}
