/*
 * solve.c -- restatement of the preconditioner and restarted GMRES (test
 * infrastructure).
 *
 *   block preconditioner setup          precond_fmm.c:147-263, 553-652
 *     (level depth-1 cubes; block[i*M+j] from panelIA0(pnlX=j, pnlY=i),
 *      read by LAPACK as column-major, plus the area diagonal)
 *   cached-LU apply                     precond_fmm.c:861-953
 *   diagonal apply                      precond_fmm.c:664-728
 *   GMRES (Templates, left-preconditioned, MGS, Givens)
 *                                       gmres.c:153-373, 527-621
 * The LU and the level-1 loops are those of oracle/blas_mini.c, which the
 * reference build in oracle/_ref/ links, so the two agree to rounding.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "internal.h"

void dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info);
void dgetrs_(char *trans, int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb,
             int *info);
double dnrm2_(const int *n, const double *x, const int *incx);
void drotg_(double *a, double *b, double *c, double *s);

typedef struct {
  or_sys *s;
  int fail;
} pc_ctx;

static void pc_build_range(void *vctx, int begin, int end) {
  pc_ctx *c = (pc_ctx *)vctx;
  or_sys *s = c->s;
  double scale1 = (1.0 + s->epsilon) / 2.0, scale2 = (1.0 + 1.0 / s->epsilon) / 2.0;
  int b, i, j;
  for (b = begin; b < end; b++) {
    int hm = s->pcSize[b], M = 2 * hm, st = s->pcStart[b], info = 0;
    double *A = (double *)calloc((size_t)M * M, sizeof(double));
    for (i = 0; i < hm; i++) {
      int Y = st + i;
      for (j = 0; j < hm; j++) {
        int X = st + j;
        double K[4];
        or_panel_ia0_raw(s, &s->pn, X, Y, K);
        A[(size_t)i * M + j] = -K[1];
        A[(size_t)i * M + j + hm] = -K[0];
        A[(size_t)(i + hm) * M + j] = -K[3];
        A[(size_t)(i + hm) * M + j + hm] = -K[2];
      }
      A[(size_t)i * M + i] += scale1 * s->pn.area[Y];
      A[(size_t)(i + hm) * M + i + hm] += scale2 * s->pn.area[Y];
    }
    s->pcPiv[b] = (int *)malloc((size_t)M * sizeof(int));
    dgetrf_(&M, &M, A, &M, s->pcPiv[b], &info);
    if (info != 0) c->fail = 1;
    s->pcLU[b] = A;
  }
}

int or_precond_setup(or_sys *s, int mode) {
  s->pcMode = mode;
  if (mode == 2) {
    int lev = s->t.depth - 1, c, b;
    pc_ctx ctx;
    s->pcLevel = lev;
    s->pcBlocks = s->t.levStart[lev + 1] - s->t.levStart[lev];
    s->pcStart = (int *)malloc((size_t)s->pcBlocks * sizeof(int));
    s->pcSize = (int *)malloc((size_t)s->pcBlocks * sizeof(int));
    s->pcLU = (double **)calloc((size_t)s->pcBlocks, sizeof(double *));
    s->pcPiv = (int **)calloc((size_t)s->pcBlocks, sizeof(int *));
    for (b = 0, c = s->t.levStart[lev]; c < s->t.levStart[lev + 1]; c++, b++) {
      s->pcStart[b] = s->t.itemStart[c];
      s->pcSize[b] = s->t.itemCount[c];
    }
    ctx.s = s; ctx.fail = 0;
    or_parallel_for(s->pcBlocks, or_thread_count(s), pc_build_range, &ctx);
    return ctx.fail ? 0 : 1;
  }
  return 1;
}

void or_precond_apply(or_sys *s, const double *b, double *x) {
  int n = s->pn.n, i, k;
  if (s->pcMode < 0) {
    memcpy(x, b, (size_t)2 * n * sizeof(double));
  } else if (s->pcMode == 2) {
    char N = 'N';
    int one = 1;
    for (k = 0; k < s->pcBlocks; k++) {
      int hm = s->pcSize[k], M = 2 * hm, st = s->pcStart[k], info = 0;
      double *rhs = (double *)malloc((size_t)M * sizeof(double));
      for (i = 0; i < hm; i++) { rhs[i] = b[st + i]; rhs[i + hm] = b[n + st + i]; }
      dgetrs_(&N, &M, &one, s->pcLU[k], &M, s->pcPiv[k], rhs, &M, &info);
      for (i = 0; i < hm; i++) { x[st + i] = rhs[i]; x[n + st + i] = rhs[i + hm]; }
      free(rhs);
    }
  } else {
    double scale1 = (1.0 + s->epsilon) / 2.0, scale2 = (1.0 + 1.0 / s->epsilon) / 2.0;
    for (i = 0; i < n; i++) {
      x[i] = b[i] / (scale1 * s->pn.area[i]);
      x[n + i] = b[n + i] / (scale2 * s->pn.area[i]);
    }
  }
}

static double ddot_n(int n, const double *x, const double *y) {
  double s = 0.0;
  int i;
  for (i = 0; i < n; i++) s += x[i] * y[i];
  return s;
}

#define BASIS_CHUNK (1 << 16)
#define BASIS_MIN_N (1 << 20)

/* gmres_basis, gmres.c:527-621 (chunked dot above BASIS_MIN_N) */
static void gmres_basis(int iter, int n, double *h, double *v, int ldv, double *w) {
  int k, i;
  int one = 1;
  for (k = 0; k < iter; k++) {
    const double *vk = &v[(size_t)k * ldv];
    double hk;
    if (n >= BASIS_MIN_N) {
      int nc = (n + BASIS_CHUNK - 1) / BASIS_CHUNK, c;
      hk = 0.0;
      for (c = 0; c < nc; c++) {
        int off = c * BASIS_CHUNK, len = n - off < BASIS_CHUNK ? n - off : BASIS_CHUNK;
        hk += ddot_n(len, w + off, vk + off);
      }
    } else {
      hk = ddot_n(n, w, vk);
    }
    h[k] = hk;
    if (-hk != 0.0) for (i = 0; i < n; i++) w[i] += (-hk) * vk[i];
  }
  h[iter] = dnrm2_(&n, w, &one);
  memcpy(&v[(size_t)iter * ldv], w, (size_t)n * sizeof(double));
  if (h[iter] > 0.0) {
    double sc = 1.0 / h[iter];
    for (i = 0; i < n; i++) v[(size_t)iter * ldv + i] *= sc;
  }
}

static void rot(double *x, double *y, double c, double sn) {
  double xv = *x, yv = *y;
  *x = c * xv + sn * yv;
  *y = c * yv - sn * xv;
}

/* gmres_update, gmres.c:364-373: y = H\s (upper), x += V y */
static void gmres_update(int it, int n, double *x, const double *h, int ldh, const double *s,
                         const double *v, int ldv) {
  double *y = (double *)malloc((size_t)(it > 0 ? it : 1) * sizeof(double));
  int i, j;
  memcpy(y, s, (size_t)it * sizeof(double));
  for (j = it - 1; j >= 0; j--) {
    if (y[j] != 0.0) {
      y[j] /= h[(size_t)j * ldh + j];
      for (i = j - 1; i >= 0; i--) y[i] -= y[j] * h[(size_t)j * ldh + i];
    }
  }
  for (j = 0; j < it; j++) {
    double t = 1.0 * y[j];
    for (i = 0; i < n; i++) x[i] += t * v[(size_t)j * ldv + i];
  }
  free(y);
}

int or_gmres(or_sys *s, const double *b, double *x, int restrt, int *iter, double *resid) {
  int n = 2 * s->pn.n, ldh = restrt + 1, maxit = *iter, i, k, one = 1;
  double tol = *resid, bnrm2, rnorm, aa, bb;
  double *r = (double *)calloc((size_t)n, sizeof(double));
  double *sv = (double *)calloc((size_t)n, sizeof(double));
  double *w = (double *)calloc((size_t)n, sizeof(double));
  double *v = (double *)calloc((size_t)n * (restrt + 1), sizeof(double));
  double *h = (double *)calloc((size_t)ldh * (restrt + 2), sizeof(double));
  double *cs = &h[(size_t)restrt * ldh], *sn = &h[(size_t)(restrt + 1) * ldh];
  int info = 0;
  memcpy(w, b, (size_t)n * sizeof(double));
  if (dnrm2_(&n, x, &one) != 0.0) {
    memcpy(w, b, (size_t)n * sizeof(double));
    or_matvec(s, -1.0, x, 1.0, w);
  }
  or_precond_apply(s, w, r);
  bnrm2 = dnrm2_(&n, b, &one);
  if (bnrm2 == 0.0) bnrm2 = 1.0;
  /* converged at the initial guess: like gmres.c:232, *iter and *resid keep
     their input values */
  if (dnrm2_(&n, r, &one) / bnrm2 < tol) goto done;
  *iter = 0;
  for (;;) {
    i = 0;
    memcpy(v, r, (size_t)n * sizeof(double));
    rnorm = dnrm2_(&n, v, &one);
    if (!(rnorm > 0.0) || rnorm != rnorm) {
      *resid = (rnorm != rnorm) ? rnorm : 0.0;
      info = (rnorm != rnorm) ? 2 : 0;
      goto done;
    }
    aa = 1.0 / rnorm;
    for (k = 0; k < n; k++) v[k] *= aa;
    sv[0] = rnorm;
    for (k = 1; k < n; k++) sv[k] = 0.0;
    for (;;) {
      double *hc;
      ++i;
      ++(*iter);
      or_matvec(s, 1.0, &v[(size_t)(i - 1) * n], 0.0, w);
      memcpy(r, w, (size_t)n * sizeof(double));
      or_precond_apply(s, r, w);
      hc = &h[(size_t)(i - 1) * ldh];
      gmres_basis(i, n, hc, v, n, w);
      for (k = 0; k < i - 1; k++) rot(&hc[k], &hc[k + 1], cs[k], sn[k]);
      aa = hc[i - 1];
      bb = hc[i];
      drotg_(&aa, &bb, &cs[i - 1], &sn[i - 1]);
      rot(&hc[i - 1], &hc[i], cs[i - 1], sn[i - 1]);
      rot(&sv[i - 1], &sv[i], cs[i - 1], sn[i - 1]);
      *resid = fabs(sv[i]) / bnrm2;
      if (*resid <= tol) {
        gmres_update(i, n, x, h, ldh, sv, v, n);
        goto done;
      }
      if (*iter == maxit || i >= restrt) break;
    }
    gmres_update(i, n, x, h, ldh, sv, v, n);
    memcpy(w, b, (size_t)n * sizeof(double));
    or_matvec(s, -1.0, x, 1.0, w);
    or_precond_apply(s, w, r);
    sv[i] = dnrm2_(&n, r, &one);
    *resid = sv[i] / bnrm2;
    if (*resid <= tol) goto done;
    if (*iter == maxit) { info = 1; goto done; }
  }
done:
  free(r); free(sv); free(w); free(v); free(h);
  return info;
}
