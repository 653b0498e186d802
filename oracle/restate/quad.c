/*
 * quad.c -- restatement of the Galerkin panel quadrature (test infrastructure).
 *
 * Follows src/numQuad.c and src/kernel.c operation by operation:
 *   Gauss-Legendre tables on [0,1]       numQuad.c:205-295
 *   kernelKER4 (the four BIE kernels)    kernel.c:109-147
 *   nrCommonVtx (exact vertex equality)  numQuad.c:312-353
 *   pnlThr0 / pnlTwo0 / pnlOne0 / pnlNil0 numQuad.c:401-618 (Sauter rules)
 *   panelIA0 (case dispatch, 4*Ax*Ay)    numQuad.c:629-697
 *   panelRHS + kernelRHS                  numQuad.c:786-819, kernel.c:152-167
 */
#include <math.h>
#include <string.h>
#include "internal.h"

/* Gauss-Legendre abscissas/weights on [0,1] as tabulated in numQuad.c:221-294
 * (15 decimals, the published values the reference uses). */
static const double kT[11][10] = {
  {0},
  {0.500000000000000},
  {0.211324865405187, 0.788675134594813},
  {0.112701665379258, 0.500000000000000, 0.887298334620742},
  {0.069431844202974, 0.330009478207572, 0.669990521792428, 0.930568155797026},
  {0.046910077030668, 0.230765344947158, 0.500000000000000, 0.769234655052841, 0.953089922969332},
  {0.033765242898424, 0.169395306766868, 0.380690406958402, 0.619309593041598, 0.830604693233132,
   0.966234757101576},
  {0.025446043828621, 0.129234407200303, 0.297077424311301, 0.500000000000000, 0.702922575688699,
   0.870765592799697, 0.974553956171379},
  {0.019855071751232, 0.101666761293187, 0.237233795041836, 0.408282678752175, 0.591717321247825,
   0.762766204958164, 0.898333238706813, 0.980144928248768},
  {0.015919880246187, 0.081984446336682, 0.193314283649705, 0.337873288298095, 0.500000000000000,
   0.662126711701904, 0.806685716350295, 0.918015553663318, 0.984080119753813},
  {0.013046735741414, 0.067468316655508, 0.160295215850488, 0.283302302935376, 0.425562830509184,
   0.574437169490816, 0.716697697064624, 0.839704784149512, 0.932531683344492, 0.986953264258586}};
static const double kW[11][10] = {
  {0},
  {1.000000000000000},
  {0.500000000000000, 0.500000000000000},
  {0.277777777777778, 0.444444444444444, 0.277777777777778},
  {0.173927422568727, 0.326072577431273, 0.326072577431273, 0.173927422568727},
  {0.118463442528095, 0.239314335249683, 0.284444444444444, 0.239314335249683, 0.118463442528095},
  {0.085662246189585, 0.180380786524070, 0.233956967286346, 0.233956967286346, 0.180380786524069,
   0.085662246189585},
  {0.064742483084435, 0.139852695744638, 0.190915025252560, 0.208979591836735, 0.190915025252559,
   0.139852695744638, 0.064742483084435},
  {0.050614268145188, 0.111190517226687, 0.156853322938944, 0.181341891689181, 0.181341891689181,
   0.156853322938944, 0.111190517226687, 0.050614268145188},
  {0.040637194180787, 0.090324080347429, 0.130305348201467, 0.156173538520002, 0.165119677500630,
   0.156173538520002, 0.130305348201468, 0.090324080347429, 0.040637194180787},
  {0.033335672154344, 0.074725674575290, 0.109543181257991, 0.134633359654998, 0.147762112357376,
   0.147762112357376, 0.134633359654998, 0.109543181257991, 0.074725674575290, 0.033335672154344}};

void or_init_quad(or_sys *s) {
  memcpy(s->tLeg, kT, sizeof(kT));
  memcpy(s->wLeg, kW, sizeof(kW));
}

void or_kernel_ker4(double kappa, double eps, const double *x, const double *nX,
                    const double *nY, double *y) {
  double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
  double r = sqrt(r2);
  double expKa = exp(-kappa * r);
  double ip0 = nX[0] * nY[0] + nX[1] * nY[1] + nX[2] * nY[2];
  double ipX = nX[0] * x[0] + nX[1] * x[1] + nX[2] * x[2];
  double ipY = nY[0] * x[0] + nY[1] * x[1] + nY[2] * x[2];
  double G0 = 1.0 / r * OR_FOURPI_I;
  double Gk = expKa * G0;
  double coef = (kappa * r + 1.0) * expKa;
  double dG0dy = ipY * G0 / r2;
  double dGkdy = coef * dG0dy;
  double dG0dx = ipX * G0 / r2;
  double dGkdx = coef * dG0dx;
  double ddG0dxdy = (ip0 * G0 - dG0dy * ipX * 3.0) / r2;
  double ddGkdxdy = coef * ddG0dxdy - kappa * kappa * expKa * ipX * dG0dy;
  y[0] = G0 - Gk;
  y[1] = eps * dGkdy - dG0dy;
  y[2] = dGkdx / eps - dG0dx;
  y[3] = ddGkdxdy - ddG0dxdy;
}

static int same3(const double *a, const double *b) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

/* nrCommonVtx, numQuad.c:312-353 (X, Y are tree indices; same index = same panel) */
static int common_vtx(const or_panels *pn, int X, int Y, int *idxX, int *idxY) {
  const double *p = &pn->vtx[9 * X], *q = &pn->vtx[9 * Y];
  int n1, n2 = 0, flag = 0, cnt = 0;
  idxX[0] = idxY[0] = 0; idxX[1] = idxY[1] = 1; idxX[2] = idxY[2] = 2;
  if (X == Y) return 3;
  for (n1 = 0; n1 < 3; n1++) {
    flag = 0;
    for (n2 = 0; n2 < 3; n2++) {
      if (same3(&p[3 * n1], &q[3 * n2])) { flag = 1; cnt++; break; }
    }
    if (flag) break;
  }
  if (!flag) return 0;
  idxX[0] = n1 % 3; idxX[1] = (n1 + 1) % 3; idxX[2] = (n1 + 2) % 3;
  idxY[0] = n2 % 3; idxY[1] = (n2 + 1) % 3; idxY[2] = (n2 + 2) % 3;
  if (same3(&p[3 * idxX[1]], &q[3 * idxY[2]])) cnt = 2;
  if (same3(&p[3 * idxX[2]], &q[3 * idxY[1]])) cnt = -2;
  return cnt;
}

typedef struct {
  double kappa, eps;
  const double *nX, *nY;
} kctx;

static void kern(const kctx *k, const double *r, double *f) {
  or_kernel_ker4(k->kappa, k->eps, r, k->nX, k->nY, f);
}

static void pnl_thr0(const or_sys *s, const kctx *kc, int q, const double *a2, const double *a0,
                     double *intgr) {
  const double *t = s->tLeg[q], *w = s->wLeg[q];
  double r1[3], r2[3], r3[3], r4[3], r5[3], r6[3];
  double f1[4], f2[4], f3[4], f4[4], f5[4], f6[4], iy_[4];
  int iy, jy, ky, ix, k, i;
  for (i = 0; i < 4; i++) intgr[i] = 0.0;
  for (iy = 0; iy < q; iy++) {
    for (jy = 0; jy < q; jy++) {
      double omg1 = t[iy] * (1.0 - t[jy]);
      for (ky = 0; ky < q; ky++) {
        for (i = 0; i < 4; i++) iy_[i] = 0.0;
        for (ix = 0; ix < q; ix++) {
          double eta1 = t[ix], fta1 = 1.0 - eta1;
          for (k = 0; k < 3; k++) {
            r1[k] = omg1 * (eta1 * a2[k] + a0[k]);
            r2[k] = omg1 * (fta1 * a0[k] - eta1 * a2[k]);
            r3[k] = omg1 * (a2[k] + eta1 * a0[k]);
            r4[k] = -omg1 * (eta1 * a2[k] + a0[k]);
            r5[k] = omg1 * (eta1 * a2[k] - fta1 * a0[k]);
            r6[k] = -omg1 * (a2[k] + eta1 * a0[k]);
          }
          kern(kc, r1, f1); kern(kc, r2, f2); kern(kc, r3, f3);
          kern(kc, r4, f4); kern(kc, r5, f5); kern(kc, r6, f6);
          for (i = 0; i < 4; i++)
            iy_[i] += (f1[i] + f3[i] + f4[i] + f2[i] + f5[i] + f6[i]) * w[ix];
        }
        for (i = 0; i < 4; i++)
          intgr[i] += iy_[i] * omg1 * (t[iy] * t[iy]) * t[jy] * w[iy] * w[jy] * w[ky];
      }
    }
  }
}

static void pnl_two0(const or_sys *s, const kctx *kc, int q, const double *a, const double *b,
                     const double *c, double *intgr) {
  const double *t = s->tLeg[q], *w = s->wLeg[q];
  double r1[3], r2[3], r3[3], r4[3], r5[3], r6[3];
  double f1[4], f2[4], f3[4], f4[4], f5[4], f6[4], iy_[4];
  int ix, jx, iy, jy, k, i;
  for (i = 0; i < 4; i++) intgr[i] = 0.0;
  for (ix = 0; ix < q; ix++) {
    for (jx = 0; jx < q; jx++) {
      double omg1 = t[ix] * t[jx];
      for (i = 0; i < 4; i++) iy_[i] = 0.0;
      for (iy = 0; iy < q; iy++) {
        double eta1 = t[iy], fta1 = 1.0 - eta1;
        for (jy = 0; jy < q; jy++) {
          double eta2 = t[jy], eta3 = eta1 * eta2, fta2 = 1.0 - eta2, fta3 = 1.0 - eta3;
          for (k = 0; k < 3; k++) {
            r1[k] = omg1 * (eta1 * (a[k] + eta2 * b[k]) + fta1 * c[k]);
            r2[k] = omg1 * (eta1 * (b[k] + eta2 * a[k]) + fta3 * c[k]);
            r3[k] = omg1 * (fta1 * a[k] + b[k] + eta3 * c[k]);
            r4[k] = omg1 * (eta1 * (eta2 * b[k] - fta2 * a[k]) + c[k]);
            r5[k] = omg1 * (eta3 * b[k] - fta3 * a[k] + eta1 * c[k]);
            r6[k] = omg1 * (eta1 * b[k] - fta1 * a[k] + eta3 * c[k]);
          }
          kern(kc, r1, f1); kern(kc, r2, f2); kern(kc, r3, f3);
          kern(kc, r4, f4); kern(kc, r5, f5); kern(kc, r6, f6);
          for (i = 0; i < 4; i++) {
            double intgrd = (f1[i] + f3[i] + f4[i] + f2[i] + f5[i] + f6[i]) * eta1;
            iy_[i] += intgrd * w[iy] * w[jy];
          }
        }
      }
      for (i = 0; i < 4; i++) intgr[i] += iy_[i] * t[jx] * (omg1 * omg1) * w[jx] * w[ix];
    }
  }
}

static void pnl_one0(const or_sys *s, const kctx *kc, int q, const double *a2, const double *a0,
                     const double *b2, const double *b0, double *intgr) {
  const double *t = s->tLeg[q], *w = s->wLeg[q];
  double r1[3], r2[3], f1[4], f2[4], iy_[4];
  int ix, iy, jy, ky, k, i;
  for (i = 0; i < 4; i++) intgr[i] = 0.0;
  for (ix = 0; ix < q; ix++) {
    double omg = t[ix];
    for (i = 0; i < 4; i++) iy_[i] = 0.0;
    for (iy = 0; iy < q; iy++) {
      double eta1 = t[iy];
      for (jy = 0; jy < q; jy++) {
        double eta2 = t[jy];
        double wij = w[iy] * w[jy] * eta1;
        for (ky = 0; ky < q; ky++) {
          double eta3 = t[ky];
          for (k = 0; k < 3; k++) {
            r1[k] = omg * (a2[k] + eta2 * a0[k] - eta1 * (b2[k] + eta3 * b0[k]));
            r2[k] = omg * (eta1 * (a2[k] + eta3 * a0[k]) - (b2[k] + eta2 * b0[k]));
          }
          kern(kc, r1, f1); kern(kc, r2, f2);
          for (i = 0; i < 4; i++) iy_[i] += (f1[i] + f2[i]) * w[ky] * wij;
        }
      }
    }
    for (i = 0; i < 4; i++) intgr[i] += iy_[i] * (omg * omg) * omg * w[ix];
  }
}

static void pnl_nil0(const or_sys *s, const kctx *kc, int q, const double *r0, const double *ax2,
                     const double *ax0, const double *ay1, const double *ay2, double *intgr) {
  const double *t = s->tLeg[q], *w = s->wLeg[q];
  double r[3], r1[3], f1[4], iy_[4];
  int ix, jx, iy, jy, k, i;
  for (i = 0; i < 4; i++) intgr[i] = 0.0;
  for (ix = 0; ix < q; ix++) {
    for (jx = 0; jx < q; jx++) {
      for (k = 0; k < 3; k++) r1[k] = r0[k] + t[ix] * (ax2[k] + t[jx] * ax0[k]);
      for (i = 0; i < 4; i++) iy_[i] = 0.0;
      for (iy = 0; iy < q; iy++) {
        for (jy = 0; jy < q; jy++) {
          for (k = 0; k < 3; k++) r[k] = r1[k] - t[iy] * (ay1[k] + t[jy] * ay2[k]);
          kern(kc, r, f1);
          for (i = 0; i < 4; i++) iy_[i] += f1[i] * t[iy] * w[iy] * w[jy];
        }
      }
      for (i = 0; i < 4; i++) intgr[i] += iy_[i] * t[ix] * w[ix] * w[jx];
    }
  }
}

/* panelIA0, numQuad.c:629-697.  X is the outer (target) panel, Y the inner. */
void or_panel_ia0_raw(const or_sys *s, const or_panels *pn, int X, int Y, double out[4]) {
  int idxX[3], idxY[3], k, i;
  int q = s->p.quad_order;
  double intgr[4], a0[3], b0[3], r0[3];
  const double *ex = &pn->edge[9 * X], *ey = &pn->edge[9 * Y];
  kctx kc;
  int nVtx = common_vtx(pn, X, Y, idxX, idxY);
  kc.kappa = s->p.kappa; kc.eps = s->epsilon;
  kc.nX = &pn->nrm[3 * X]; kc.nY = &pn->nrm[3 * Y];
  if (nVtx == 0) {
    for (k = 0; k < 3; k++) r0[k] = pn->vtx[9 * X + k] - pn->vtx[9 * Y + k];
    pnl_nil0(s, &kc, q, r0, &ex[6], &ex[0], &ey[6], &ey[0], intgr);
  } else if (nVtx == 1) {
    pnl_one0(s, &kc, q, &ex[3 * idxX[2]], &ex[3 * idxX[0]], &ey[3 * idxY[2]], &ey[3 * idxY[0]], intgr);
  } else if (nVtx == 2) {
    pnl_two0(s, &kc, q, &ex[3 * idxX[2]], &ex[3 * idxX[0]], &ey[3 * idxY[0]], intgr);
  } else if (nVtx == -2) {
    for (k = 0; k < 3; k++) { b0[k] = -ey[3 * idxY[0] + k]; a0[k] = -ex[3 * idxX[0] + k]; }
    pnl_two0(s, &kc, q, &ex[3 * idxX[1]], b0, a0, intgr);
  } else {
    pnl_thr0(s, &kc, q, &ex[6], &ex[0], intgr);
  }
  for (i = 0; i < 4; i++) out[i] = 4.0 * pn->area[X] * pn->area[Y] * intgr[i];
}

/* panelRHS + kernelRHS (numQuad.c:786-819, kernel.c:152-167) */
void or_panel_rhs(const or_sys *s, int X, const double *chr, double out[2]) {
  int q = s->p.quad_order, ix, jx, k;
  const double *t = s->tLeg[q], *w = s->wLeg[q];
  const double *v0 = &s->pn.vtx[9 * X], *ax2 = &s->pn.edge[9 * X + 6], *ax0 = &s->pn.edge[9 * X];
  const double *n = &s->pn.nrm[3 * X];
  double r0[3], r[3];
  for (k = 0; k < 3; k++) r0[k] = v0[k] - chr[k];
  out[0] = out[1] = 0.0;
  for (ix = 0; ix < q; ix++) {
    for (jx = 0; jx < q; jx++) {
      double r2, ri, r3i, ip;
      for (k = 0; k < 3; k++) r[k] = r0[k] + t[ix] * (ax2[k] + t[jx] * ax0[k]);
      r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      ri = 1.0 / sqrt(r2);
      r3i = ri / r2;
      ip = n[0] * r[0] + n[1] * r[1] + n[2] * r[2];
      out[0] += ri * t[ix] * w[ix] * w[jx];
      out[1] += (-ip * r3i) * t[ix] * w[ix] * w[jx];
    }
  }
  out[0] *= 2.0 * s->pn.area[X];
  out[1] *= 2.0 * s->pn.area[X];
}
