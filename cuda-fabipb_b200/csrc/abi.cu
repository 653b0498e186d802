// abi.cu -- the reference's GPU plugin ABI (include/gpu_backend.h) on top of
// the device context.  A host built from the reference sources links this
// library in place of its src/gpu_backend_cuda.cu.
//
// The ABI passes the host's `struct ssystem *` (layout: include/
// fabipb_host_abi.h) and host vectors indexed by pnl->idx.  On the first call
// for a system the backend builds its own device context from the panels in
// tree order (sys->pnlLst), then checks that its octree, leaf layout, near
// pairs and M2L pairs are identical to the ones the host built in gkInit /
// setupFMM (src/gkSetup.c:446, src/fmm.c:430); any difference is reported
// as a failure rather than computed on a different tree.
//
// Physics parameters the ABI does not pass (kappa, epsilon, epsilon1; the
// charge-tree thetas and orders) are read from the host's own globals and
// functions through weak references, as the reference backend reads them
// (src/gpu/gpu_backend_cuda_internal.h:20-42).
#include <mutex>
#include <string>

#include "../../include/fabipb_host_abi.h"
#include "../../include/gpu_backend.h"
#include "context.cuh"

extern "C" {
extern double kappa __attribute__((weak));
extern double epsilon __attribute__((weak));
extern double epsilon1 __attribute__((weak));
double energyTreeTheta(void) __attribute__((weak));
double rhsTreeTheta(void) __attribute__((weak));
int rhsChargeExpansionOrder(struct ssystem *sys, int level) __attribute__((weak));
extern double fmmNearGpuKernelTime __attribute__((weak));
}

namespace fb {

bool abi_disjoint_pairs(const double *vtx, const double *nrm, const double *area, long long nPairs,
                        const int *dst, const int *src, double kappa, double eps, double *k0, double *k1,
                        double *k2, double *k3, int *done, cudaStream_t s);
bool abi_coulomb_dot(Context &c, const double *rhs, const double *sgm, double eps1, double *dot);
bool launch_energy_mode(Context &c, const double *sgm, int mode, double *raw_host);

namespace {

char g_nearErr[1024] = "";
char g_m2lErr[1024] = "";
std::mutex g_mu;

struct AbiState {
  const ssystem *sys = nullptr;
  Context *ctx = nullptr;
  const ssystem *denseSys = nullptr;
  Context *dense = nullptr;
  bool pending = false;        // device expansions hold this matvec's locals
  const ssystem *chargeSys = nullptr;
};
AbiState g;

void near_err(const char *m) { snprintf(g_nearErr, sizeof(g_nearErr), "%s", m); }
void m2l_err(const char *m) { snprintf(g_m2lErr, sizeof(g_m2lErr), "%s", m); }

bool host_physics(double *kap, double *eps, double *eps1) {
  if (&kappa == nullptr || &epsilon == nullptr || &epsilon1 == nullptr) {
    set_error("host globals kappa/epsilon/epsilon1 are not linked into this process");
    return false;
  }
  *kap = kappa;
  *eps = epsilon;
  *eps1 = epsilon1;
  return true;
}

// (order, orderMom) of getOrders (src/gkSetup.c:42-81) from the level arrays
void host_orders(const ssystem *sys, int *order, int *orderMom) {
  const int d = sys->depth, h = sys->height;
  bool fixed = true;
  for (int l = h; l <= d; l++)
    if (sys->ordM2L[l] != sys->maxOrder || sys->ordMom[l] != sys->maxOrder) fixed = false;
  if (fixed && (d == h || sys->ordM2L[h] == sys->ordM2L[d])) {
    *order = sys->maxOrder;
    *orderMom = 0;
    return;
  }
  *order = -sys->ordM2L[d];
  *orderMom = (sys->ordMom[d] == sys->maxOrder && sys->ordMom[h] == sys->maxOrder && d > h)
                  ? -1
                  : sys->ordMom[d] - sys->ordM2L[d];
}

void gather_panels(const ssystem *sys, std::vector<double> &vtx, std::vector<double> &nrm,
                   std::vector<double> &area) {
  const int n = sys->nPnls;
  vtx.resize(9 * (size_t)n);
  nrm.resize(3 * (size_t)n);
  area.resize(n);
  int i = 0;
  for (const panel *p = sys->pnlLst; p != nullptr && i < n; p = p->nextC, i++) {
    for (int k = 0; k < 3; k++)
      for (int c = 0; c < 3; c++) vtx[9 * (size_t)i + 3 * k + c] = p->vtx[k][c];
    for (int c = 0; c < 3; c++) nrm[3 * (size_t)i + c] = p->normal[c];
    area[i] = p->area;
  }
}

bool same_tree(const ssystem *sys, const Context &c) {
  const PanelTree &pt = c.pt;
  if (pt.nLeaves != sys->nLeafCubesFlat || (int)pt.nearSrc.size() != sys->nNearPairsFlat ||
      (int)pt.m2lPairSrc.size() != sys->nM2LPairsFlat || pt.nFmm != sys->nFmmCubesFlat) {
    set_error("device octree differs from the host's (leaves %d/%d near %zu/%d m2l %zu/%d cubes %d/%d)",
              pt.nLeaves, sys->nLeafCubesFlat, pt.nearSrc.size(), sys->nNearPairsFlat, pt.m2lPairSrc.size(),
              sys->nM2LPairsFlat, pt.nFmm, sys->nFmmCubesFlat);
    return false;
  }
  for (int L = 0; L < pt.nLeaves; L++)
    if (pt.leafStart[L] != sys->leafPanelStart[L] || pt.leafCount[L] != sys->leafPanelCount[L]) {
      set_error("device leaf layout differs from the host's at leaf %d", L);
      return false;
    }
  for (size_t k = 0; k < pt.nearSrc.size(); k++)
    if (pt.nearSrc[k] != sys->nearPairSrc[k] || pt.nearDst[k] != sys->nearPairDst[k]) {
      set_error("device near-pair list differs from the host's at %zu", k);
      return false;
    }
  for (size_t k = 0; k < pt.m2lPairSrc.size(); k++)
    if (pt.m2lPairSrc[k] != sys->m2lPairSrc[k] || pt.m2lPairDst[k] != sys->m2lPairDst[k]) {
      set_error("device M2L list differs from the host's at %zu", k);
      return false;
    }
  return true;
}

Context *build_context(const ssystem *sys, bool dense) {
  double kap, eps, eps1;
  if (!host_physics(&kap, &eps, &eps1)) return nullptr;
  fabipb_b200_params p;
  fabipb_b200_default_params(&p);
  host_orders(sys, &p.order, &p.order_mom);
  p.depth = sys->depth;
  p.height = sys->height;
  p.quad_order = sys->maxQuadOrder;
  p.sep_ratio = sys->maxSepRatio;
  p.kappa = kap;
  p.eps1 = eps1;
  p.eps2 = eps * eps1;
  const char *pe = getenv("FABIPB_B200_PRECISION");
  p.precision = (pe && std::string(pe) == "mixed") ? FABIPB_B200_MIXED : FABIPB_B200_FP64;
  if (&rhsTreeTheta != nullptr) p.rhs_theta = rhsTreeTheta();
  if (&energyTreeTheta != nullptr) p.energy_theta = energyTreeTheta();
  std::vector<double> vtx, nrm, area;
  gather_panels(sys, vtx, nrm, area);
  void *h = nullptr;
  if (!create_context(&p, sys->nPnls, vtx.data(), nrm.data(), area.data(), dense, &h)) return nullptr;
  Context *c = (Context *)h;
  // the reference host evaluates -p with epsilon = eps2/eps1 exactly
  c->epsilon = eps;
  if (!dense && !same_tree(sys, *c)) {
    fabipb_b200_destroy(c);
    return nullptr;
  }
  for (int l = 0; l <= sys->depth; l++)
    if (l >= sys->height && (c->pt.ordM2L[l] != sys->ordM2L[l] || c->pt.ordMom[l] != sys->ordMom[l])) {
      set_error("expansion orders differ from the host's at level %d", l);
      fabipb_b200_destroy(c);
      return nullptr;
    }
  return c;
}

Context *ctx_for(ssystem *sys) {
  if (g.sys == sys && g.ctx) return g.ctx;
  if (g.ctx) fabipb_b200_destroy(g.ctx);
  g.ctx = nullptr;
  g.sys = nullptr;
  g.pending = false;
  g.chargeSys = nullptr;
  Context *c = build_context(sys, false);
  if (!c) return nullptr;
  g.ctx = c;
  g.sys = sys;
  return c;
}

bool ensure_charges(Context &c, ssystem *sys) {
  if (g.chargeSys == sys && c.ct != nullptr) return true;
  if (sys->nChar <= 0 || sys->pos == nullptr || sys->chr == nullptr) {
    set_error("system has no charges");
    return false;
  }
  c.chargeOrders.clear();
  if (&rhsChargeExpansionOrder != nullptr)
    for (int l = 0; l <= sys->depth; l++) c.chargeOrders.push_back(l >= sys->height ? rhsChargeExpansionOrder(sys, l) : 0);
  if (!setup_charges(c, sys->nChar, sys->pos, sys->chr)) return false;
  g.chargeSys = sys;
  return true;
}

bool h2d(Context &c, double *d, const double *h, size_t n) {
  FB_CUDA(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  return true;
}
bool d2h(Context &c, double *h, const double *d, size_t n) {
  FB_CUDA(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  FB_CUDA(cudaStreamSynchronize(c.stream));
  return true;
}

}  // namespace
}  // namespace fb

using namespace fb;

extern "C" {

int gpuBackendAvailable(void) {
  int n = 0;
  return (cudaGetDeviceCount(&n) == cudaSuccess && n > 0) ? 1 : 0;
}

const char *gpuNearfieldLastError(void) { return g_nearErr[0] ? g_nearErr : "unknown nearfield GPU failure"; }

const char *gpuM2LLastError(void) { return g_m2lErr[0] ? g_m2lErr : "unknown M2L GPU failure"; }

int gpuNearfieldApply(struct ssystem *sys, double alpha, const double *sgm, double *pot) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sgm == nullptr || pot == nullptr) { near_err("invalid input pointer"); return 0; }
  Context *c = ctx_for(sys);
  if (!c) { near_err(get_error()); return 0; }
  const size_t n2 = 2 * (size_t)c->n;
  bool ok = h2d(*c, c->d_x, sgm, n2) && h2d(*c, c->d_y, pot, n2) && launch_near(*c, c->d_x, alpha, c->d_y) &&
            d2h(*c, pot, c->d_y, n2);
  if (!ok) near_err(get_error());
  return ok ? 1 : 0;
}

int gpuDirectApply(struct ssystem *sys, double alpha, double beta, const double *sgm, double *pot) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sgm == nullptr || pot == nullptr) return 0;
  if (g.denseSys != sys || g.dense == nullptr) {
    if (g.dense) fabipb_b200_destroy(g.dense);
    g.dense = build_context(sys, true);
    g.denseSys = g.dense ? sys : nullptr;
    if (!g.dense) { near_err(get_error()); return 0; }
  }
  Context *c = g.dense;
  const size_t n2 = 2 * (size_t)c->n;
  bool ok = h2d(*c, c->d_x, sgm, n2) && h2d(*c, c->d_y, pot, n2) &&
            op_apply(*c, FABIPB_B200_NEAR, alpha, c->d_x, beta, c->d_y) && d2h(*c, pot, c->d_y, n2);
  if (!ok) near_err(get_error());
  return ok ? 1 : 0;
}

int gpuQ2MApply(struct ssystem *sys, const double *sgm) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sgm == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { m2l_err(get_error()); return 0; }
  g.pending = false;
  bool ok = h2d(*c, c->d_x, sgm, 2 * (size_t)c->n) && launch_far_upward(*c, c->d_x);
  if (ok) ok = cudaStreamSynchronize(c->stream) == cudaSuccess;
  if (!ok) { m2l_err(get_error()); return 0; }
  g.pending = true;
  return 1;
}

int gpuM2LApply(struct ssystem *sys) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sys->nM2LPairsFlat <= 0) { m2l_err("invalid input or empty M2L pair list"); return 0; }
  Context *c = ctx_for(sys);
  if (!c) { m2l_err(get_error()); return 0; }
  if (g.pending) return 1;  // locals already on the device (see gpuQ2MApply)
  // host moments in, M2L on the device, host locals out (overwritten)
  const int NM = c->NM, nF = c->pt.nFmm;
  const size_t plane = (size_t)nF * NM;
  std::vector<double> mom(2 * plane, 0.0), lec(4 * plane, 0.0);
  for (int f = 0; f < nF; f++) {
    const cube *cb = sys->fmmCubeByIdx[f];
    int nm = nmom(sys->ordMom[cb->level]);
    for (int e = 0; e < nm && e < NM; e++) {
      mom[(size_t)f * NM + e] = cb->mom_pot[e];
      mom[plane + (size_t)f * NM + e] = cb->mom_dpdn[e];
    }
  }
  bool ok = h2d(*c, c->d_mom, mom.data(), 2 * plane) &&
            cudaMemsetAsync(c->d_lec, 0, 4 * plane * sizeof(double), c->stream) == cudaSuccess &&
            launch_m2l_only(*c) && d2h(*c, lec.data(), c->d_lec, 4 * plane);
  if (!ok) { m2l_err(get_error()); return 0; }
  for (int f = 0; f < nF; f++) {
    cube *cb = sys->fmmCubeByIdx[f];
    int nm = nmom(sys->ordMom[cb->level]);
    for (int e = 0; e < nm && e < NM; e++) {
      cb->lec_k1[e] = lec[(size_t)f * NM + e];
      cb->lec_k2[e] = lec[plane + (size_t)f * NM + e];
      cb->lec_k3[e] = lec[2 * plane + (size_t)f * NM + e];
      cb->lec_k4[e] = lec[3 * plane + (size_t)f * NM + e];
    }
  }
  return 1;
}

int gpuL2PApply(struct ssystem *sys, double alpha, double beta, double *pot) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || pot == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { m2l_err(get_error()); return 0; }
  const size_t n2 = 2 * (size_t)c->n;
  bool ok = true;
  if (!g.pending) {
    // local expansions come from the host leaf cubes
    const int NM = c->NM, nF = c->pt.nFmm;
    const size_t plane = (size_t)nF * NM;
    std::vector<double> lec(4 * plane, 0.0);
    int L = 0;
    for (const cube *cb = sys->cubeList[sys->depth]; cb != nullptr; cb = cb->next, L++) {
      int f = c->pt.cubeFmm[c->pt.leafCube[L]];
      int nm = nmom(sys->ordMom[cb->level]);
      for (int e = 0; e < nm && e < NM; e++) {
        lec[(size_t)f * NM + e] = cb->lec_k1[e];
        lec[plane + (size_t)f * NM + e] = cb->lec_k2[e];
        lec[2 * plane + (size_t)f * NM + e] = cb->lec_k3[e];
        lec[3 * plane + (size_t)f * NM + e] = cb->lec_k4[e];
      }
    }
    ok = h2d(*c, c->d_lec, lec.data(), 4 * plane);
  }
  g.pending = false;
  ok = ok && h2d(*c, c->d_y, pot, n2) && launch_l2p(*c, alpha, beta, c->d_y, nullptr, 0.0, 0.0) &&
       d2h(*c, pot, c->d_y, n2);
  if (!ok) { m2l_err(get_error()); return 0; }
  return 1;
}

void gpuReleaseMatvecCaches(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  // keep the charge tree if it lives in the same context: release only the
  // dense operator and reset the pipeline state
  if (g.dense) fabipb_b200_destroy(g.dense);
  g.dense = nullptr;
  g.denseSys = nullptr;
  g.pending = false;
}

void gpuReleaseChargeTreeCache(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g.ctx) free_charges(*g.ctx);
  g.chargeSys = nullptr;
}

int gpuSetupRHS(struct ssystem *sys, int qOrder, double fac, double *sgm) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sgm == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { near_err(get_error()); return 0; }
  if (qOrder != c->prm.quad_order) { near_err("quadrature order differs from the system's"); return 0; }
  c->rhsFac = fac;
  bool ok = ensure_charges(*c, sys) && launch_rhs(*c, 0, c->d_y) && d2h(*c, sgm, c->d_y, 2 * (size_t)c->n);
  c->rhsFac = 0.0;
  if (!ok) { near_err(get_error()); return 0; }
  return 1;
}

int gpuChargeTreeRHS(struct ssystem *sys, int qOrder, double fac, double *sgm) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sgm == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { near_err(get_error()); return 0; }
  if (qOrder != c->prm.quad_order) { near_err("quadrature order differs from the system's"); return 0; }
  c->rhsFac = fac;
  bool ok = ensure_charges(*c, sys) && launch_rhs(*c, 1, c->d_y) && d2h(*c, sgm, c->d_y, 2 * (size_t)c->n);
  c->rhsFac = 0.0;
  if (!ok) { near_err(get_error()); return 0; }
  return 1;
}

int gpuPanelChargeTreeEnergy(struct ssystem *sys, const double *sgm, double *pot) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || sgm == nullptr || pot == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { near_err(get_error()); return 0; }
  bool ok = ensure_charges(*c, sys) && h2d(*c, c->d_x, sgm, 2 * (size_t)c->n) &&
            launch_energy_mode(*c, c->d_x, 1, pot);
  if (!ok) { near_err(get_error()); return 0; }
  return 1;
}

int gpuRhsReuseCoulombDot(struct ssystem *sys, const double *rhs, const double *sgm, double *dot) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || rhs == nullptr || sgm == nullptr || dot == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { near_err(get_error()); return 0; }
  const size_t n2 = 2 * (size_t)c->n;
  bool ok = h2d(*c, c->d_x, sgm, n2) && h2d(*c, c->d_w, rhs, n2) &&
            abi_coulomb_dot(*c, c->d_w, c->d_x, c->prm.eps1, dot);
  if (!ok) { near_err(get_error()); return 0; }
  return 1;
}

int gpuRhsReusePanelChargeTreeEnergy(struct ssystem *sys, const double *rhs, const double *sgm, double *pot) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || rhs == nullptr || sgm == nullptr || pot == nullptr) return 0;
  Context *c = ctx_for(sys);
  if (!c) { near_err(get_error()); return 0; }
  const size_t n2 = 2 * (size_t)c->n;
  double dot = 0.0, scr = 0.0;
  bool ok = ensure_charges(*c, sys) && h2d(*c, c->d_x, sgm, n2) && h2d(*c, c->d_w, rhs, n2) &&
            abi_coulomb_dot(*c, c->d_w, c->d_x, c->prm.eps1, &dot) && launch_energy_mode(*c, c->d_x, 2, &scr);
  if (!ok) { near_err(get_error()); return 0; }
  *pot = dot + scr;
  return 1;
}

int gpuBuildPrecondPairsBatched(struct ssystem *sys, const int *pairSrc, const int *pairDst, long long nPairs,
                                double *k0, double *k1, double *k2, double *k3) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (sys == nullptr || pairSrc == nullptr || pairDst == nullptr || nPairs <= 0) return 0;
  if (k0 == nullptr || k1 == nullptr || k2 == nullptr || k3 == nullptr) return 0;
  double kap, eps, eps1;
  if (!host_physics(&kap, &eps, &eps1)) { near_err(get_error()); return 0; }
  std::vector<double> vtx, nrm, area;
  gather_panels(sys, vtx, nrm, area);  // indexed by pnl->idx (tree order)
  bool ok = abi_disjoint_pairs(vtx.data(), nrm.data(), area.data(), nPairs, pairDst, pairSrc, kap, eps, k0, k1, k2,
                               k3, nullptr, 0);
  if (!ok) { near_err(get_error()); return 0; }
  return 1;
}

int gpuBuildPrecondDisjointBlock(struct panel **panels, int nPanels, const int *dstLocal, const int *srcLocal,
                                 int nPairs, double *block) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (panels == nullptr || dstLocal == nullptr || srcLocal == nullptr || block == nullptr || nPanels <= 0 ||
      nPairs <= 0)
    return 0;
  double kap, eps, eps1;
  if (!host_physics(&kap, &eps, &eps1)) { near_err(get_error()); return 0; }
  std::vector<double> vtx(9 * (size_t)nPanels), nrm(3 * (size_t)nPanels), area(nPanels);
  for (int i = 0; i < nPanels; i++) {
    const panel *p = panels[i];
    for (int k = 0; k < 3; k++)
      for (int c = 0; c < 3; c++) vtx[9 * (size_t)i + 3 * k + c] = p->vtx[k][c];
    for (int c = 0; c < 3; c++) nrm[3 * (size_t)i + c] = p->normal[c];
    area[i] = p->area;
  }
  std::vector<double> k0(nPairs), k1(nPairs), k2(nPairs), k3(nPairs);
  std::vector<int> done(nPairs, 0);
  if (!abi_disjoint_pairs(vtx.data(), nrm.data(), area.data(), nPairs, dstLocal, srcLocal, kap, eps, k0.data(),
                          k1.data(), k2.data(), k3.data(), done.data(), 0)) {
    near_err(get_error());
    return 0;
  }
  const int hm = nPanels, M = 2 * hm;
  for (int i = 0; i < nPairs; i++) {
    if (!done[i]) continue;
    const int d = dstLocal[i], s = srcLocal[i];
    block[(size_t)d * M + s] = -k1[i];
    block[(size_t)d * M + s + hm] = -k0[i];
    block[(size_t)(d + hm) * M + s] = -k3[i];
    block[(size_t)(d + hm) * M + s + hm] = -k2[i];
  }
  return 1;
}

}  // extern "C"
