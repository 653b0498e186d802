// quad.cuh -- FP64 Galerkin panel quadrature on the device.
//
// The singular and near-singular panel pairs (shared vertex, shared edge,
// self) stay in double precision.  These functions evaluate the reference's
// rules for them:
//   kernelKER4                     src/kernel.c:109-147
//   nrCommonVtx (exact equality)   src/numQuad.c:312-353
//   pnlOne0 / pnlTwo0 / pnlThr0    src/numQuad.c:401-571 (Sauter's
//                                  transformations to regular integrals)
//   pnlNil0                        src/numQuad.c:586-618
//   panelIA0                       src/numQuad.c:629-697 (4*Ax*Ay*integral)
// and the one-point (q=1) disjoint rule the near-field kernel evaluates on
// the fly, K = Ax*Ay*KER4(mX - mY) with m = v0 + (v1-v0)/2 + (v2-v1)/4.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace fb {

// Gauss-Legendre abscissas/weights on [0,1] for orders 1..10 (the published
// 15-decimal values of src/numQuad.c:221-294), filled by init_quad_tables().
// The library is one translation unit (fabipb_b200.cu), so the constant
// tables are defined here once.
__constant__ double c_tLeg[11][10];
__constant__ double c_wLeg[11][10];
bool init_quad_tables();

struct PanelD {
  double v[3][3];   // vertices
  double a[3][3];   // a[0]=v2-v1, a[1]=v0-v2, a[2]=v1-v0 (input.c:743-747)
  double n[3];      // unit normal
  double area;
};

__device__ __forceinline__ void ker4_d(double kappa, double eps, const double *x, const double *nX,
                                       const double *nY, double *y) {
  double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x[0], x[0]), __dmul_rn(x[1], x[1])), __dmul_rn(x[2], x[2]));
  double r = sqrt(r2);
  double expKa = exp(-kappa * r);
  double ip0 = nX[0] * nY[0] + nX[1] * nY[1] + nX[2] * nY[2];
  double ipX = nX[0] * x[0] + nX[1] * x[1] + nX[2] * x[2];
  double ipY = nY[0] * x[0] + nY[1] * x[1] + nY[2] * x[2];
  double G0 = 1.0 / r * kFourPiI;
  double Gk = expKa * G0;
  double coef = (kappa * r + 1.0) * expKa;
  double dG0dy = ipY * G0 / r2;
  double dGkdy = coef * dG0dy;
  double dG0dx = ipX * G0 / r2;
  double dGkdx = coef * dG0dx;
  double ddG0 = (ip0 * G0 - dG0dy * ipX * 3.0) / r2;
  double ddGk = coef * ddG0 - kappa * kappa * expKa * ipX * dG0dy;
  y[0] = G0 - Gk;
  y[1] = eps * dGkdy - dG0dy;
  y[2] = dGkdx / eps - dG0dx;
  y[3] = ddGk - ddG0;
}

__device__ __forceinline__ bool same3(const double *a, const double *b) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

// nrCommonVtx: 3 same panel, 0 disjoint, 1 one vertex, 2 / -2 shared edge
__device__ inline int common_vtx(const PanelD &p, const PanelD &q, bool samePanel, int *ix, int *iy) {
  ix[0] = iy[0] = 0; ix[1] = iy[1] = 1; ix[2] = iy[2] = 2;
  if (samePanel) return 3;
  int n1, n2 = 0, flag = 0, cnt = 0;
  for (n1 = 0; n1 < 3; n1++) {
    flag = 0;
    for (n2 = 0; n2 < 3; n2++) {
      if (same3(p.v[n1], q.v[n2])) { flag = 1; cnt++; break; }
    }
    if (flag) break;
  }
  if (!flag) return 0;
  ix[0] = n1 % 3; ix[1] = (n1 + 1) % 3; ix[2] = (n1 + 2) % 3;
  iy[0] = n2 % 3; iy[1] = (n2 + 1) % 3; iy[2] = (n2 + 2) % 3;
  if (same3(p.v[ix[1]], q.v[iy[2]])) cnt = 2;
  if (same3(p.v[ix[2]], q.v[iy[1]])) cnt = -2;
  return cnt;
}

struct KerCtx {
  double kappa, eps;
  const double *nX, *nY;
};

__device__ inline void pnl_thr0_d(const KerCtx &k, int q, const double *a2, const double *a0, double *I) {
  const double *t = c_tLeg[q], *w = c_wLeg[q];
  for (int i = 0; i < 4; i++) I[i] = 0.0;
  for (int iy = 0; iy < q; iy++)
    for (int jy = 0; jy < q; jy++) {
      double omg1 = t[iy] * (1.0 - t[jy]);
      for (int ky = 0; ky < q; ky++) {
        double Y[4] = {0, 0, 0, 0};
        for (int ix = 0; ix < q; ix++) {
          double eta1 = t[ix], fta1 = 1.0 - eta1;
          double r[6][3], f[6][4];
          for (int c = 0; c < 3; c++) {
            r[0][c] = omg1 * (eta1 * a2[c] + a0[c]);
            r[1][c] = omg1 * (fta1 * a0[c] - eta1 * a2[c]);
            r[2][c] = omg1 * (a2[c] + eta1 * a0[c]);
            r[3][c] = -omg1 * (eta1 * a2[c] + a0[c]);
            r[4][c] = omg1 * (eta1 * a2[c] - fta1 * a0[c]);
            r[5][c] = -omg1 * (a2[c] + eta1 * a0[c]);
          }
          for (int s = 0; s < 6; s++) ker4_d(k.kappa, k.eps, r[s], k.nX, k.nY, f[s]);
          for (int i = 0; i < 4; i++)
            Y[i] += (f[0][i] + f[2][i] + f[3][i] + f[1][i] + f[4][i] + f[5][i]) * w[ix];
        }
        for (int i = 0; i < 4; i++) I[i] += Y[i] * omg1 * (t[iy] * t[iy]) * t[jy] * w[iy] * w[jy] * w[ky];
      }
    }
}

__device__ inline void pnl_two0_d(const KerCtx &k, int q, const double *a, const double *b,
                                  const double *cc, double *I) {
  const double *t = c_tLeg[q], *w = c_wLeg[q];
  for (int i = 0; i < 4; i++) I[i] = 0.0;
  for (int ix = 0; ix < q; ix++)
    for (int jx = 0; jx < q; jx++) {
      double omg1 = t[ix] * t[jx];
      double Y[4] = {0, 0, 0, 0};
      for (int iy = 0; iy < q; iy++) {
        double eta1 = t[iy], fta1 = 1.0 - eta1;
        for (int jy = 0; jy < q; jy++) {
          double eta2 = t[jy], eta3 = eta1 * eta2, fta2 = 1.0 - eta2, fta3 = 1.0 - eta3;
          double r[6][3], f[6][4];
          for (int c = 0; c < 3; c++) {
            r[0][c] = omg1 * (eta1 * (a[c] + eta2 * b[c]) + fta1 * cc[c]);
            r[1][c] = omg1 * (eta1 * (b[c] + eta2 * a[c]) + fta3 * cc[c]);
            r[2][c] = omg1 * (fta1 * a[c] + b[c] + eta3 * cc[c]);
            r[3][c] = omg1 * (eta1 * (eta2 * b[c] - fta2 * a[c]) + cc[c]);
            r[4][c] = omg1 * (eta3 * b[c] - fta3 * a[c] + eta1 * cc[c]);
            r[5][c] = omg1 * (eta1 * b[c] - fta1 * a[c] + eta3 * cc[c]);
          }
          for (int s = 0; s < 6; s++) ker4_d(k.kappa, k.eps, r[s], k.nX, k.nY, f[s]);
          for (int i = 0; i < 4; i++) {
            double v = (f[0][i] + f[2][i] + f[3][i] + f[1][i] + f[4][i] + f[5][i]) * eta1;
            Y[i] += v * w[iy] * w[jy];
          }
        }
      }
      for (int i = 0; i < 4; i++) I[i] += Y[i] * t[jx] * (omg1 * omg1) * w[jx] * w[ix];
    }
}

__device__ inline void pnl_one0_d(const KerCtx &k, int q, const double *a2, const double *a0,
                                  const double *b2, const double *b0, double *I) {
  const double *t = c_tLeg[q], *w = c_wLeg[q];
  for (int i = 0; i < 4; i++) I[i] = 0.0;
  for (int ix = 0; ix < q; ix++) {
    double omg = t[ix];
    double Y[4] = {0, 0, 0, 0};
    for (int iy = 0; iy < q; iy++) {
      double eta1 = t[iy];
      for (int jy = 0; jy < q; jy++) {
        double eta2 = t[jy], wij = w[iy] * w[jy] * eta1;
        for (int ky = 0; ky < q; ky++) {
          double eta3 = t[ky], r1[3], r2[3], f1[4], f2[4];
          for (int c = 0; c < 3; c++) {
            r1[c] = omg * (a2[c] + eta2 * a0[c] - eta1 * (b2[c] + eta3 * b0[c]));
            r2[c] = omg * (eta1 * (a2[c] + eta3 * a0[c]) - (b2[c] + eta2 * b0[c]));
          }
          ker4_d(k.kappa, k.eps, r1, k.nX, k.nY, f1);
          ker4_d(k.kappa, k.eps, r2, k.nX, k.nY, f2);
          for (int i = 0; i < 4; i++) Y[i] += (f1[i] + f2[i]) * w[ky] * wij;
        }
      }
    }
    for (int i = 0; i < 4; i++) I[i] += Y[i] * (omg * omg) * omg * w[ix];
  }
}

__device__ inline void pnl_nil0_d(const KerCtx &k, int q, const double *r0, const double *ax2,
                                  const double *ax0, const double *ay1, const double *ay2, double *I) {
  const double *t = c_tLeg[q], *w = c_wLeg[q];
  for (int i = 0; i < 4; i++) I[i] = 0.0;
  for (int ix = 0; ix < q; ix++)
    for (int jx = 0; jx < q; jx++) {
      double r1[3], Y[4] = {0, 0, 0, 0};
      for (int c = 0; c < 3; c++) r1[c] = r0[c] + t[ix] * (ax2[c] + t[jx] * ax0[c]);
      for (int iy = 0; iy < q; iy++)
        for (int jy = 0; jy < q; jy++) {
          double r[3], f[4];
          for (int c = 0; c < 3; c++) r[c] = r1[c] - t[iy] * (ay1[c] + t[jy] * ay2[c]);
          ker4_d(k.kappa, k.eps, r, k.nX, k.nY, f);
          for (int i = 0; i < 4; i++) Y[i] += f[i] * t[iy] * w[iy] * w[jy];
        }
      for (int i = 0; i < 4; i++) I[i] += Y[i] * t[ix] * w[ix] * w[jx];
    }
}

// panelIA0 for outer panel X, inner panel Y; returns the case in *caseOut
__device__ inline void panel_ia0_d(int q, double kappa, double eps, const PanelD &X, const PanelD &Y,
                                   bool samePanel, double out[4], int *caseOut) {
  int ix[3], iy[3];
  double I[4];
  KerCtx k{kappa, eps, X.n, Y.n};
  int nv = common_vtx(X, Y, samePanel, ix, iy);
  if (nv == 0) {
    double r0[3];
    for (int c = 0; c < 3; c++) r0[c] = X.v[0][c] - Y.v[0][c];
    pnl_nil0_d(k, q, r0, X.a[2], X.a[0], Y.a[2], Y.a[0], I);
  } else if (nv == 1) {
    pnl_one0_d(k, q, X.a[ix[2]], X.a[ix[0]], Y.a[iy[2]], Y.a[iy[0]], I);
  } else if (nv == 2) {
    pnl_two0_d(k, q, X.a[ix[2]], X.a[ix[0]], Y.a[iy[0]], I);
  } else if (nv == -2) {
    double b0[3], a0[3];
    for (int c = 0; c < 3; c++) { b0[c] = -Y.a[iy[0]][c]; a0[c] = -X.a[ix[0]][c]; }
    pnl_two0_d(k, q, X.a[ix[1]], b0, a0, I);
  } else {
    pnl_thr0_d(k, q, X.a[2], X.a[0], I);
  }
  for (int i = 0; i < 4; i++) out[i] = 4.0 * X.area * Y.area * I[i];
  if (caseOut) *caseOut = nv;
}

}  // namespace fb
