/*
 * expan.c -- restatement of the Cartesian Taylor FMM (test infrastructure).
 *
 *   index tables mkIndex/initExpan        expan.c:39-129
 *   radial derivatives kernelDG0DGk       kernel.c:84-104 (and the Coulomb-only
 *                                          recurrence of treecode.c:283-347)
 *   Cartesian derivative tensor           expan.c:138-209 (setupDerivs)
 *   leaf moments / noments                moments.c:363-543 (calcMoments0)
 *   M2M / M2L / L2L convolutions          expan.c:223-494
 *   applyFMM pass order and L2P/Q2M dgemv fmm.c:710-838
 *   near field by destination leaf        fmm.c:554-593
 *   MtVmain (D - K with the beta trick)   fabipb.c:1237-1287
 *
 * Q2M/L2P use the same column loops as the reference's dgemv_ when it is
 * linked against oracle/blas_mini.c, so the two agree to the last bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "internal.h"

void or_init_expan(or_sys *s) {
  int order = s->maxOrder, deriv = order + 1, nd = or_nmom(deriv);
  int k, n, k1, k2, i, sgn = 1, nn;
  s->idxDim = order + 3;
  s->idx3 = (int *)calloc((size_t)s->idxDim * s->idxDim * s->idxDim, sizeof(int));
  for (i = nn = 0; nn <= deriv; nn++)
    for (k1 = 0; k1 <= nn; k1++)
      for (k2 = 0; k2 <= nn - k1; k2++, i++)
        s->idx3[(k1 * s->idxDim + k2) * s->idxDim + (nn - k1 - k2)] = i;
  s->fact = (double *)calloc((size_t)order + 4, sizeof(double));
  s->ifact = (double *)calloc((size_t)order + 4, sizeof(double));
  s->ifact3 = (double *)calloc((size_t)nd, sizeof(double));
  s->sgn3 = (int *)calloc((size_t)nd, sizeof(int));
  s->fact[0] = s->ifact[0] = 1.0;
  for (k = 1; k <= order + 3; k++) { s->fact[k] = s->fact[k - 1] * k; s->ifact[k] = 1.0 / s->fact[k]; }
  for (k = n = 0; n <= deriv; n++, sgn *= -1)
    for (k1 = 0; k1 <= n; k1++)
      for (k2 = 0; k2 <= n - k1; k2++, k++) {
        int k3 = n - k1 - k2;
        double f3 = s->fact[k1] * s->fact[k2] * s->fact[k3];
        s->ifact3[k] = 1.0 / f3;
        s->sgn3[k] = sgn;
      }
}

/*
 * D^alpha G0 and D^alpha Gk at x for |alpha| <= order into d0/dk (length
 * nMom(order)).  Work arrays hold one row per derivative level p as in
 * setupDerivs; coulombOnly skips Gk (setupCoulombDerivsLocal).
 */
void or_setup_derivs(const or_sys *s, int order, const double *x, double *d0, double *dk,
                     int coulombOnly) {
  int P = order, stride = or_nmom(P), p, p1, iRow, iRow1, i1, i2, i3, idx, idx1, idx2, k;
  double *g0 = (double *)malloc((size_t)(P + 2) * stride * sizeof(double));
  double *gk = (double *)malloc((size_t)(P + 2) * stride * sizeof(double));
  double G0[64], Gk[64];
  double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  double kappa = s->p.kappa;
#define D0(pp, ii) g0[(pp) * stride + (ii)]
#define DK(pp, ii) gk[(pp) * stride + (ii)]
  if (coulombOnly) {
    double r2 = -1.0 / (r * r);
    G0[0] = OR_FOURPI_I / r;
    for (k = 0; k < P; k++) G0[k + 1] = (2 * k + 1) * r2 * G0[k];
  } else {
    double rexp = exp(-kappa * r), r1 = 1.0 / r, rr2 = r1 * r1, nr2 = -rr2, kappa2 = kappa * kappa;
    G0[0] = r1 * OR_FOURPI_I;
    Gk[0] = rexp * G0[0];
    G0[1] = nr2 * G0[0];
    Gk[1] = -Gk[0] * (rr2 + kappa * r1);
    for (k = 1; k < P; k++) {
      G0[k + 1] = (2 * k + 1) * nr2 * G0[k];
      Gk[k + 1] = rr2 * (kappa2 * Gk[k - 1] - (2 * k + 1) * Gk[k]);
    }
  }
  for (p = 0; p <= P; p++) { D0(p, 0) = G0[p]; if (!coulombOnly) DK(p, 0) = Gk[p]; }
  for (p = 0; p < P; p++) {
    p1 = p + 1;
    D0(p, 1) = D0(p1, 0) * x[2]; D0(p, 2) = D0(p1, 0) * x[1]; D0(p, 3) = D0(p1, 0) * x[0];
    if (!coulombOnly) {
      DK(p, 1) = DK(p1, 0) * x[2]; DK(p, 2) = DK(p1, 0) * x[1]; DK(p, 3) = DK(p1, 0) * x[0];
    }
  }
  for (iRow = 2; iRow <= P; iRow++) {
    for (p = 0; p <= P - iRow; p++) {
      p1 = p + 1;
      idx = or_idx3(s, 0, 0, iRow);
      iRow1 = iRow - 1;
      idx1 = or_idx3(s, 0, 0, iRow1);
      idx2 = or_idx3(s, 0, 0, iRow - 2);
      D0(p, idx) = D0(p1, idx1) * x[2] + D0(p1, idx2) * iRow1;
      if (!coulombOnly) DK(p, idx) = DK(p1, idx1) * x[2] + DK(p1, idx2) * iRow1;
      idx++;
      idx1 = or_idx3(s, 0, 0, iRow1);
      D0(p, idx) = D0(p1, idx1) * x[1];
      if (!coulombOnly) DK(p, idx) = DK(p1, idx1) * x[1];
      idx++;
      for (i2 = 2; i2 <= iRow; i2++, idx++) {
        i3 = iRow - i2;
        idx1 = or_idx3(s, 0, i2 - 1, i3);
        idx2 = or_idx3(s, 0, i2 - 2, i3);
        D0(p, idx) = D0(p1, idx1) * x[1] + D0(p1, idx2) * (i2 - 1);
        if (!coulombOnly) DK(p, idx) = DK(p1, idx1) * x[1] + DK(p1, idx2) * (i2 - 1);
      }
      for (i2 = 0; i2 <= iRow1; i2++, idx++) {
        i3 = iRow1 - i2;
        idx1 = or_idx3(s, 0, i2, i3);
        D0(p, idx) = D0(p1, idx1) * x[0];
        if (!coulombOnly) DK(p, idx) = DK(p1, idx1) * x[0];
      }
      for (i1 = 2; i1 <= iRow; i1++) {
        for (i2 = 0; i2 <= iRow - i1; i2++, idx++) {
          i3 = iRow - i1 - i2;
          idx1 = or_idx3(s, i1 - 1, i2, i3);
          idx2 = or_idx3(s, i1 - 2, i2, i3);
          D0(p, idx) = D0(p1, idx1) * x[0] + D0(p1, idx2) * (i1 - 1);
          if (!coulombOnly) DK(p, idx) = DK(p1, idx1) * x[0] + DK(p1, idx2) * (i1 - 1);
        }
      }
    }
  }
  memcpy(d0, g0, (size_t)stride * sizeof(double));
  if (!coulombOnly) memcpy(dk, gk, (size_t)stride * sizeof(double));
#undef D0
#undef DK
  free(g0);
  free(gk);
}

/* setupConVect, moments.c:390-410: convVec[alpha] = trns^alpha / alpha! */
static void con_vect(const or_sys *s, int order, const double *trns, double *cv) {
  double f1[64], f2[64], f3[64];
  int i, n, i1, i2;
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
}

/* convolution, moments.c:363-385 (c = a * b, overwrite) */
static void convolve(const or_sys *s, int order, const double *a, const double *b, double *c) {
  int i, n, i1, i2, i3, k1, k2, k3;
  for (i = n = 0; n <= order; n++)
    for (i1 = 0; i1 <= n; i1++)
      for (i2 = 0; i2 <= n - i1; i2++, i++) {
        double tmp = 0.0;
        i3 = n - i1 - i2;
        for (k1 = 0; k1 <= i1; k1++)
          for (k2 = 0; k2 <= i2; k2++)
            for (k3 = 0; k3 <= i3; k3++)
              tmp += a[or_idx3(s, i1 - k1, i2 - k2, i3 - k3)] * b[or_idx3(s, k1, k2, k3)];
        c[i] = tmp;
      }
}

/*
 * calcOneMoment0 / calcOneNoment / calcMoments0 (moments.c:422-543).  The
 * file-scope scratch vectors of the reference carry stale top-order entries
 * into the job==1 convolution; only entries below the top order are read by
 * calcOneNoment, so fresh zeroed scratch gives the same noments.
 */
static void leaf_moments(or_sys *s, int leaf, int order, int job, double *M) {
  int nMom = or_nmom(order), start = s->leafStart[leaf], cnt = s->leafCount[leaf];
  int c = s->t.levStart[s->t.depth] + leaf, idx, i, n, i1, i2;
  const double *ctr = &s->t.x[3 * c];
  double *cv1 = (double *)calloc((size_t)nMom, sizeof(double));
  double *cv2 = (double *)calloc((size_t)nMom, sizeof(double));
  double *buf = (double *)calloc((size_t)nMom, sizeof(double));
  double *loc = (double *)calloc((size_t)nMom, sizeof(double));
  double *tr = (double *)calloc((size_t)nMom, sizeof(double));
  for (idx = 0; idx < cnt; idx++) {
    int P = start + idx, order1 = (job == 0) ? order : order - 1;
    const double *v0 = &s->pn.vtx[9 * P], *v1 = v0 + 3, *v2 = v0 + 6, *nrm = &s->pn.nrm[3 * P];
    double a1[3], a2[3], trns[3], area2 = 2.0 * s->pn.area[P];
    double *mb = (job == 0) ? loc : buf;
    for (i = 0; i < 3; i++) { a1[i] = v1[i] - v0[i]; a2[i] = v2[i] - v0[i]; }
    memset(cv1, 0, (size_t)nMom * sizeof(double));
    memset(cv2, 0, (size_t)nMom * sizeof(double));
    con_vect(s, order1, a1, cv1);
    con_vect(s, order1, a2, cv2);
    for (i = n = 0; n <= order1; n++)
      for (i1 = 0; i1 <= n; i1++)
        for (i2 = 0; i2 <= n - i1; i2++, i++) { cv1[i] *= s->fact[n]; cv2[i] *= s->fact[n]; }
    convolve(s, order, cv1, cv2, mb);
    for (i = n = 0; n <= order; n++)
      for (i1 = 0; i1 <= n; i1++)
        for (i2 = 0; i2 <= n - i1; i2++, i++) mb[i] *= area2 * s->ifact[n + 2];
    if (job == 1) {
      for (i = 0; i < nMom; i++) loc[i] = 0.0;
      for (i = n = 0; n < order; n++)
        for (i1 = 0; i1 <= n; i1++)
          for (i2 = 0; i2 <= n - i1; i2++, i++) {
            int i3 = n - i1 - i2;
            loc[or_idx3(s, i1 + 1, i2, i3)] += nrm[0] * buf[i];
            loc[or_idx3(s, i1, i2 + 1, i3)] += nrm[1] * buf[i];
            loc[or_idx3(s, i1, i2, i3 + 1)] += nrm[2] * buf[i];
          }
    }
    for (i = 0; i < 3; i++) trns[i] = v0[i] - ctr[i];
    con_vect(s, order, trns, tr);
    convolve(s, order, tr, loc, &M[(size_t)idx * nMom]);
  }
  free(cv1); free(cv2); free(buf); free(loc); free(tr);
}

/* setupFMM, fmm.c:430-524: leaf matrices, expansion storage, layouts */
void or_setup_fmm(or_sys *s) {
  or_tree *t = &s->t;
  int depth = t->depth, height = t->height, lev, c, idx, L;
  long long off = 0;
  s->nLeaves = t->levStart[depth + 1] - t->levStart[depth];
  s->leafStart = (int *)malloc((size_t)s->nLeaves * sizeof(int));
  s->leafCount = (int *)malloc((size_t)s->nLeaves * sizeof(int));
  for (L = 0; L < s->nLeaves; L++) {
    c = t->levStart[depth] + L;
    s->leafStart[L] = t->itemStart[c];
    s->leafCount[L] = t->itemCount[c];
  }
  /* buildApplyLayout, fmm.c:234-268 */
  s->nNear = 0;
  for (L = 0; L < s->nLeaves; L++) s->nNear += t->nNbr1[t->levStart[depth] + L];
  s->nearSrc = (int *)malloc((size_t)s->nNear * sizeof(int));
  s->nearDst = (int *)malloc((size_t)s->nNear * sizeof(int));
  s->nearOff = (int *)malloc((size_t)(s->nLeaves + 1) * sizeof(int));
  for (idx = 0, L = 0; L < s->nLeaves; L++) {
    int cc = t->levStart[depth] + L, k;
    s->nearOff[L] = idx;
    for (k = 0; k < t->nNbr1[cc]; k++, idx++) {
      s->nearSrc[idx] = t->nbr[t->nbrStart[cc] + k] - t->levStart[depth];
      s->nearDst[idx] = L;
    }
  }
  s->nearOff[s->nLeaves] = idx;
  /* buildFmmCubeLayout, fmm.c:295-324 */
  s->cubeFmm = (int *)malloc((size_t)t->nCubes * sizeof(int));
  for (c = 0; c < t->nCubes; c++) s->cubeFmm[c] = -1;
  s->nFmm = t->levStart[depth + 1] - t->levStart[height];
  s->fmmCube = (int *)malloc((size_t)s->nFmm * sizeof(int));
  for (idx = 0, lev = depth; lev >= height; lev--)
    for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++, idx++) {
      s->fmmCube[idx] = c;
      s->cubeFmm[c] = idx;
    }
  /* buildM2LPairList, fmm.c:326-373 */
  s->nM2L = 0;
  for (c = t->levStart[height]; c < t->levStart[depth + 1]; c++) s->nM2L += t->nNbr2[c] - t->nNbr1[c];
  s->m2lSrc = (int *)malloc((size_t)(s->nM2L > 0 ? s->nM2L : 1) * sizeof(int));
  s->m2lDst = (int *)malloc((size_t)(s->nM2L > 0 ? s->nM2L : 1) * sizeof(int));
  for (idx = 0, lev = depth; lev >= height; lev--)
    for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++) {
      int i;
      for (i = t->nNbr2[c] - 1; i >= t->nNbr1[c]; i--, idx++) {
        s->m2lSrc[idx] = s->cubeFmm[t->nbr[t->nbrStart[c] + i]];
        s->m2lDst[idx] = s->cubeFmm[c];
      }
    }
  /* leaf matrices (calcMoments0 with order ordMom[depth]) */
  s->nMomLeaf = or_nmom(s->ordMom[depth]);
  s->leafMatOff = (long long *)malloc((size_t)(s->nLeaves + 1) * sizeof(long long));
  for (L = 0; L < s->nLeaves; L++) { s->leafMatOff[L] = off; off += (long long)s->nMomLeaf * s->leafCount[L]; }
  s->leafMatOff[s->nLeaves] = off;
  s->Q2M0 = (double *)malloc((size_t)off * sizeof(double));
  s->Q2M1 = (double *)malloc((size_t)off * sizeof(double));
  for (L = 0; L < s->nLeaves; L++) {
    leaf_moments(s, L, s->ordMom[depth], 0, &s->Q2M0[s->leafMatOff[L]]);
    leaf_moments(s, L, s->ordMom[depth], 1, &s->Q2M1[s->leafMatOff[L]]);
  }
  s->nMomMax = or_nmom(s->maxOrder);
  s->momPot = (double *)calloc((size_t)s->nFmm * s->nMomMax, sizeof(double));
  s->momDpdn = (double *)calloc((size_t)s->nFmm * s->nMomMax, sizeof(double));
  s->lec1 = (double *)calloc((size_t)s->nFmm * s->nMomMax, sizeof(double));
  s->lec2 = (double *)calloc((size_t)s->nFmm * s->nMomMax, sizeof(double));
  s->lec3 = (double *)calloc((size_t)s->nFmm * s->nMomMax, sizeof(double));
  s->lec4 = (double *)calloc((size_t)s->nFmm * s->nMomMax, sizeof(double));
}

/* transM2MWs + convM2M, expan.c:223-247, 342-382 */
static void trans_m2m(or_sys *s, int kidC, int parC, double *cvR, double *cv1, double *cv2) {
  int ordIn = s->ordMom[s->t.level[kidC]], ordOut = s->ordMom[s->t.level[parC]];
  int nIn = or_nmom(ordIn), nOut = or_nmom(ordOut), fi = s->cubeFmm[kidC], fo = s->cubeFmm[parC];
  int i, n, i1, i2, i3, k1, k2, k3;
  double trns[3];
  double *outP = &s->momPot[(size_t)fo * s->nMomMax], *outD = &s->momDpdn[(size_t)fo * s->nMomMax];
  for (i = 0; i < 3; i++) trns[i] = s->t.x[3 * kidC + i] - s->t.x[3 * parC + i];
  con_vect(s, ordOut, trns, cvR);
  memcpy(cv1, &s->momPot[(size_t)fi * s->nMomMax], (size_t)nIn * sizeof(double));
  memcpy(cv2, &s->momDpdn[(size_t)fi * s->nMomMax], (size_t)nIn * sizeof(double));
  for (i = nIn; i < nOut; i++) { cv1[i] = 0.0; cv2[i] = 0.0; }
  for (i = n = 0; n <= ordOut; n++)
    for (i1 = 0; i1 <= n; i1++)
      for (i2 = 0; i2 <= n - i1; i2++, i++) {
        double t1 = 0.0, t2 = 0.0;
        i3 = n - i1 - i2;
        for (k1 = 0; k1 <= i1; k1++)
          for (k2 = 0; k2 <= i2; k2++)
            for (k3 = 0; k3 <= i3; k3++) {
              double a = cvR[or_idx3(s, i1 - k1, i2 - k2, i3 - k3)];
              int b = or_idx3(s, k1, k2, k3);
              t1 += a * cv1[b];
              t2 += a * cv2[b];
            }
        outP[i] += t1;
        outD[i] += t2;
      }
}

/* transL2LWs + convL2L, expan.c:295-326, 403-452 */
static void trans_l2l(or_sys *s, int parC, int kidC, double *cvR) {
  int ordIn = s->ordMom[s->t.level[parC]], ordOut = s->ordMom[s->t.level[kidC]];
  int fi = s->cubeFmm[parC], fo = s->cubeFmm[kidC];
  size_t M = (size_t)s->nMomMax;
  const double *I1 = &s->lec1[fi * M], *I2 = &s->lec2[fi * M], *I3 = &s->lec3[fi * M], *I4 = &s->lec4[fi * M];
  double *O1 = &s->lec1[fo * M], *O2 = &s->lec2[fo * M], *O3 = &s->lec3[fo * M], *O4 = &s->lec4[fo * M];
  double trns[3];
  int i, j, n, m, i1, i2, i3, j1, j2, j3;
  for (i = 0; i < 3; i++) trns[i] = s->t.x[3 * kidC + i] - s->t.x[3 * parC + i];
  con_vect(s, ordIn, trns, cvR);
  for (i = n = 0; n <= ordOut; n++)
    for (i1 = 0; i1 <= n; i1++)
      for (i2 = 0; i2 <= n - i1; i2++, i++) {
        double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
        i3 = n - i1 - i2;
        for (j = m = 0; m <= ordIn - n; m++)
          for (j1 = 0; j1 <= m; j1++)
            for (j2 = 0; j2 <= m - j1; j2++, j++) {
              int q;
              j3 = m - j1 - j2;
              q = or_idx3(s, i1 + j1, i2 + j2, i3 + j3);
              t1 += cvR[j] * I1[q];
              t2 += cvR[j] * I2[q];
              t3 += cvR[j] * I3[q];
              t4 += cvR[j] * I4[q];
            }
        O1[i] += t1; O2[i] += t2; O3[i] += t3; O4[i] += t4;
      }
}

/* transM2L + convM2L, expan.c:258-290, 471-494 */
static void trans_m2l(or_sys *s, int srcF, int dstF, const double *G0, const double *Gk,
                      double *c1, double *c2, double *v1, double *v2, double *v3) {
  int srcC = s->fmmCube[srcF], order = s->ordM2L[s->t.level[srcC]], nMom = or_nmom(order);
  size_t M = (size_t)s->nMomMax;
  const double *mp = &s->momPot[srcF * M], *md = &s->momDpdn[srcF * M];
  double *l1 = &s->lec1[dstF * M], *l2 = &s->lec2[dstF * M], *l3 = &s->lec3[dstF * M], *l4 = &s->lec4[dstF * M];
  double eps = s->epsilon;
  int i, j, n, m, i1, i2, i3, j1, j2, j3;
  for (i = 0; i < nMom; i++) {
    c1[i] = s->sgn3[i] * mp[i];
    c2[i] = s->sgn3[i] * md[i];
    v1[i] = G0[i] - Gk[i];
    v2[i] = eps * Gk[i] - G0[i];
    v3[i] = G0[i] - Gk[i] / eps;
  }
  for (i = n = 0; n <= order; n++)
    for (i1 = 0; i1 <= n; i1++)
      for (i2 = 0; i2 <= n - i1; i2++, i++) {
        double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
        i3 = n - i1 - i2;
        for (j = m = 0; m <= order - n; m++)
          for (j1 = 0; j1 <= m; j1++)
            for (j2 = 0; j2 <= m - j1; j2++, j++) {
              int q;
              j3 = m - j1 - j2;
              q = or_idx3(s, i1 + j1, i2 + j2, i3 + j3);
              t1 += c2[j] * v1[q];
              t2 += c1[j] * v2[q];
              t3 += c2[j] * v3[q];
              t4 += c1[j] * (-v1[q]);
            }
        l1[i] += t1; l2[i] += t2; l3[i] += t3; l4[i] += t4;
      }
}

/* dgemv 'N' and 'T' with the column loops of oracle/blas_mini.c */
static void gemv_n_acc(int m, int n, const double *A, const double *x, double *y) {
  int i, j;
  for (j = 0; j < n; j++) {
    double t = 1.0 * x[j];
    for (i = 0; i < m; i++) y[i] += t * A[(size_t)j * m + i];
  }
}

static void gemv_t(int m, int n, double alpha, const double *A, const double *x, double beta, double *y) {
  int i, j;
  if (m == 0 || n == 0 || (alpha == 0.0 && beta == 1.0)) return;
  if (beta != 1.0)
    for (j = 0; j < n; j++) y[j] = (beta == 0.0) ? 0.0 : beta * y[j];
  if (alpha == 0.0) return;
  for (j = 0; j < n; j++) {
    double t = 0.0;
    for (i = 0; i < m; i++) t += A[(size_t)j * m + i] * x[i];
    y[j] += alpha * t;
  }
}

/* far field only: Q2M, M2M, M2L, L2L, L2P with pot = beta*pot + alpha*K_far*sgm */
void or_far_apply(or_sys *s, double alpha, const double *sgm, double beta, double *pot) {
  or_tree *t = &s->t;
  int depth = t->depth, height = t->height, n = s->pn.n, L, lev, c, k, idx;
  size_t M = (size_t)s->nMomMax, tot = (size_t)s->nFmm * M;
  int nm = s->nMomLeaf;
  double *cvR = (double *)calloc(M + 64, sizeof(double));
  double *cv1 = (double *)calloc(M + 64, sizeof(double));
  double *cv2 = (double *)calloc(M + 64, sizeof(double));
  double *v1 = (double *)calloc(M + 64, sizeof(double));
  double *v2 = (double *)calloc(M + 64, sizeof(double));
  double *v3 = (double *)calloc(M + 64, sizeof(double));
  double *G0 = (double *)calloc(M + 64, sizeof(double));
  double *Gk = (double *)calloc(M + 64, sizeof(double));
  memset(s->momPot, 0, tot * sizeof(double)); memset(s->momDpdn, 0, tot * sizeof(double));
  memset(s->lec1, 0, tot * sizeof(double)); memset(s->lec2, 0, tot * sizeof(double));
  memset(s->lec3, 0, tot * sizeof(double)); memset(s->lec4, 0, tot * sizeof(double));
  /* Q2M: mom_pot = Q2M1 sigma_pot, mom_dpdn = Q2M0 sigma_dpdn (fmm.c:745-753) */
  for (L = 0; L < s->nLeaves; L++) {
    int f = s->cubeFmm[t->levStart[depth] + L];
    gemv_n_acc(nm, s->leafCount[L], &s->Q2M1[s->leafMatOff[L]], &sgm[s->leafStart[L]], &s->momPot[f * M]);
    gemv_n_acc(nm, s->leafCount[L], &s->Q2M0[s->leafMatOff[L]], &sgm[s->leafStart[L] + n], &s->momDpdn[f * M]);
  }
  for (lev = depth - 1; lev >= height; lev--)
    for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++)
      for (k = 0; k < t->kidCount[c]; k++) trans_m2m(s, t->kidStart[c] + k, c, cvR, cv1, cv2);
  for (idx = 0; idx < s->nM2L; idx++) {
    int sf = s->m2lSrc[idx], df = s->m2lDst[idx];
    int sc = s->fmmCube[sf], dc = s->fmmCube[df];
    double r[3];
    int order = s->ordM2L[t->level[dc]];
    for (k = 0; k < 3; k++) r[k] = t->x[3 * dc + k] - t->x[3 * sc + k];
    or_setup_derivs(s, order, r, G0, Gk, 0);
    trans_m2l(s, sf, df, G0, Gk, cv1, cv2, v1, v2, v3);
  }
  for (lev = height; lev < depth; lev++)
    for (c = t->levStart[lev]; c < t->levStart[lev + 1]; c++)
      for (k = 0; k < t->kidCount[c]; k++) trans_l2l(s, c, t->kidStart[c] + k, cvR);
  /* L2P (fmm.c:815-828) */
  for (L = 0; L < s->nLeaves; L++) {
    int f = s->cubeFmm[t->levStart[depth] + L], st = s->leafStart[L], cnt = s->leafCount[L];
    gemv_t(nm, cnt, alpha, &s->Q2M0[s->leafMatOff[L]], &s->lec1[f * M], beta, &pot[st]);
    gemv_t(nm, cnt, alpha, &s->Q2M0[s->leafMatOff[L]], &s->lec2[f * M], 1.0, &pot[st]);
    gemv_t(nm, cnt, alpha, &s->Q2M1[s->leafMatOff[L]], &s->lec3[f * M], beta, &pot[st + n]);
    gemv_t(nm, cnt, alpha, &s->Q2M1[s->leafMatOff[L]], &s->lec4[f * M], 1.0, &pot[st + n]);
  }
  free(cvR); free(cv1); free(cv2); free(v1); free(v2); free(v3); free(G0); free(Gk);
}

typedef struct {
  or_sys *s;
  double alpha;
  const double *sgm;
  double *pot;
} near_ctx;

/* nearApplyLeafStrided, fmm.c:554-593 */
static void near_range(void *vctx, int begin, int end) {
  near_ctx *c = (near_ctx *)vctx;
  or_sys *s = c->s;
  int n = s->pn.n, L, i, pr, j;
  for (L = begin; L < end; L++) {
    for (i = 0; i < s->leafCount[L]; i++) {
      int X = s->leafStart[L] + i;
      double sumPot = 0.0, sumDpdn = 0.0;
      for (pr = s->nearOff[L]; pr < s->nearOff[L + 1]; pr++) {
        int sl = s->nearSrc[pr];
        for (j = 0; j < s->leafCount[sl]; j++) {
          int Y = s->leafStart[sl] + j;
          double K[4], xp = c->sgm[Y], xd = c->sgm[Y + n];
          or_panel_ia0_raw(s, &s->pn, X, Y, K);
          sumPot += (K[0] * xd + K[1] * xp) * c->alpha;
          sumDpdn += (K[2] * xd + K[3] * xp) * c->alpha;
        }
      }
      c->pot[X] += sumPot;
      c->pot[X + n] += sumDpdn;
    }
  }
}

void or_near_apply(or_sys *s, double alpha, const double *sgm, double *pot) {
  near_ctx c;
  c.s = s; c.alpha = alpha; c.sgm = sgm; c.pot = pot;
  or_parallel_for(s->nLeaves, or_thread_count(s), near_range, &c);
}

void or_fmm_apply(or_sys *s, double alpha, const double *sgm, double beta, double *pot) {
  or_far_apply(s, alpha, sgm, beta, pot);
  or_near_apply(s, alpha, sgm, pot);
}

/* MtVmain, fabipb.c:1237-1287: y = alpha*(D - K) x + beta*y */
void or_matvec(or_sys *s, double alpha, const double *x, double beta, double *y) {
  int n = s->pn.n, i;
  double scale1 = (1.0 + s->epsilon) / 2.0 * alpha;
  double scale2 = (1.0 + 1.0 / s->epsilon) / 2.0 * alpha;
  or_fmm_apply(s, alpha, x, -beta, y);
  for (i = 0; i < n; i++) {
    y[i] = (scale1 * s->pn.area[i] * x[i] - y[i]);
    y[i + n] = scale2 * s->pn.area[i] * x[i + n] - y[i + n];
  }
}
