// charges.cu -- right-hand side and solvation energy on the device.
//
//   direct RHS      setupRHS direct loop, src/fabipb.c:788-798, with the
//                   panel quadrature of panelRHS/kernelRHS,
//                   src/numQuad.c:786-819, src/kernel.c:152-167
//   charge octree   buildChargeTree, src/chargeTree.c:228-307 (same cell
//                   tests as the panel tree, over the charge bounding cube)
//   charge moments  computeChgMoments, src/chargeTree.c:314-416
//   cluster order   rhsChargeExpansionOrder, src/chargeTree.c:117-129
//   tree RHS walk   rhsTreeWalkLocal, src/treecode.c:283-450
//   energy walk     energyTreeWalk/panelEnergyTree, src/treecode.c:581-695,
//                   summed as in panelEnergyWorker, src/treecode.c:869-887
//
// Each walk gives every panel point the reference's depth-first recursion
// and its summation order (children in index order); a warp walks its 32
// points together with one stack of (cube, lane mask) entries.  Accepted
// clusters evaluate the Cartesian derivative tensor to order p+1 (unrolled
// into registers) and contract it with the cluster moments; leaves sum their
// charges directly.  FP64, or FP32 terms with FP64 sums in mixed contexts;
// the energy is reduced per block and then in block order, so it is
// deterministic.
#include <algorithm>
#include <cstring>
#include <functional>
#include <thread>
#include <utility>

#include "context.cuh"
#include "quad.cuh"

namespace fb {

struct ChargeTreeDev {
  bool built = false;
  int nCubes = 0, depth = 0, height = 0, maxStack = 0;
  DevArena arena;
  double *d_pos = nullptr, *d_chr = nullptr;   // in charge-tree leaf order
  double *d_ctr = nullptr, *d_rad = nullptr;
  int *d_level = nullptr, *d_kidStart = nullptr, *d_kidCount = nullptr;
  int *d_itemStart = nullptr, *d_itemCount = nullptr, *d_order = nullptr;
  void *d_smom = nullptr;   // nCubes x NM signed moments (-1)^|i| M_i, FP32 in mixed contexts
  double *d_partial = nullptr;                 // energy partial sums
  int partialCap = 0;
  double *d_posOrig = nullptr, *d_chrOrig = nullptr;  // input order (direct RHS)
  float4 *d_chgF = nullptr;   // FP32 (position - root box centre, charge), mixed contexts
};

void free_charges(Context &c) {
  if (c.ct) {
    c.ct->arena.release();
    delete c.ct;
    c.ct = nullptr;
  }
}

bool setup_charges(Context &c, int m, const double *pos, const double *q) {
  free_charges(c);
  c.nChar = m;
  c.h_pos.assign(pos, pos + 3 * (size_t)m);
  c.h_chr.assign(q, q + m);
  c.ct = new ChargeTreeDev();
  if (!c.ct->arena.upload(&c.ct->d_posOrig, c.h_pos, c.stream) ||
      !c.ct->arena.upload(&c.ct->d_chrOrig, c.h_chr, c.stream))
    return false;
  return true;
}

// charge-tree Taylor order of a level (chargeTree.c:117-129)
static int charge_order(const Context &c, int level) {
  if (!c.chargeOrders.empty()) return std::min(c.chargeOrders[level], c.P);
  int order;
  if (c.prm.charge_order > 0) order = c.prm.charge_order;
  else order = std::max(c.pt.ordMom[level], 4);
  return std::min(order, c.P);
}

static bool build_charge_tree(Context &c) {
  ChargeTreeDev &d = *c.ct;
  if (d.built) return true;
  StageTimer tm("charges", c.stream);
  const int m = c.nChar;
  const double *pos = c.h_pos.data();
  double cminx = pos[0], cmaxx = pos[0], cminy = pos[1], cmaxy = pos[1], cminz = pos[2], cmaxz = pos[2];
  for (int j = 1; j < m; j++) {
    double x = pos[3 * (size_t)j], y = pos[3 * (size_t)j + 1], z = pos[3 * (size_t)j + 2];
    cminx = cminx > x ? x : cminx; cmaxx = x > cmaxx ? x : cmaxx;
    cminy = cminy > y ? y : cminy; cmaxy = y > cmaxy ? y : cmaxy;
    cminz = cminz > z ? z : cminz; cmaxz = z > cmaxz ? z : cmaxz;
  }
  double length = (cmaxx - cminx) > (cmaxy - cminy) ? (cmaxx - cminx) : (cmaxy - cminy);
  length = (cmaxz - cminz) > length ? (cmaxz - cminz) : length;
  if (length <= 0.0) length = 1.0;
  Octree t;
  std::vector<int> sorted;
  if (!build_octree(t, m, pos, c.pt.t.depth, c.pt.t.height, cminx, cminy, cminz, length, sorted)) return false;
  octree_boxes_points(t, pos, sorted);
  d.nCubes = t.nCubes;
  d.depth = t.depth;
  d.height = t.height;
  d.maxStack = 7 * t.depth + 2;
  const int NM = c.NM;
  std::vector<int> order(t.nCubes, 0);
  for (int cc = 0; cc < t.nCubes; cc++) order[cc] = (t.level[cc] >= t.height) ? charge_order(c, t.level[cc]) : 0;
  // moments (computeChgLeafMoments / transM2Mchr), host FP64
  std::vector<double> mom((size_t)t.nCubes * NM, 0.0);
  std::vector<int> mi;  // multi-indices for orders <= P
  std::vector<int> idx3((c.P + 2) * (c.P + 2) * (c.P + 2), 0);
  std::vector<double> ifact3;
  {
    double fact[32];
    fact[0] = 1.0;
    for (int k = 1; k < 32; k++) fact[k] = fact[k - 1] * k;
    int D = c.P + 2, i = 0;
    for (int n = 0; n <= c.P; n++)
      for (int a = 0; a <= n; a++)
        for (int b = 0; b <= n - a; b++, i++) {
          int cc = n - a - b;
          idx3[(a * D + b) * D + cc] = i;
          mi.push_back(a); mi.push_back(b); mi.push_back(cc);
          ifact3.push_back(1.0 / (fact[a] * fact[b] * fact[cc]));
        }
  }
  const int D = c.P + 2;
  auto conv_vect = [&](int ord, const double *tr, double *cv) {
    double f1[32], f2[32], f3[32];
    f1[0] = f2[0] = f3[0] = 1.0;
    for (int i = 1; i <= ord; i++) {
      f1[i] = f1[i - 1] * tr[0]; f2[i] = f2[i - 1] * tr[1]; f3[i] = f3[i - 1] * tr[2];
    }
    int nmo = nmom(ord);
    for (int i = 0; i < nmo; i++) {
      cv[i] = f1[mi[3 * i]] * f2[mi[3 * i + 1]] * f3[mi[3 * i + 2]];
      cv[i] *= ifact3[i];
    }
  };
  // a cube's moments depend only on its own charges or children: the cubes of a level on the
  // host's cores, each summed in the same order whatever the split
  auto per_cube = [NM](int c0, int c1, const std::function<void(int, int, double *)> &f) {
    const int nth = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int nc = c1 - c0;
    if (nc < 64 || nth == 1) {
      std::vector<double> cv(NM);
      f(c0, c1, cv.data());
      return;
    }
    std::vector<std::thread> pool;
    for (int th = 0; th < nth; th++)
      pool.emplace_back([&, th] {
        std::vector<double> cv(NM);
        f(c0 + (int)((long long)nc * th / nth), c0 + (int)((long long)nc * (th + 1) / nth), cv.data());
      });
    for (auto &th : pool) th.join();
  };
  per_cube(t.levStart[t.depth], t.levStart[t.depth + 1], [&](int a, int b, double *cv) {
    for (int cc = a; cc < b; cc++) {
      int ord = order[cc], nmo = nmom(ord);
      for (int k = 0; k < t.itemCount[cc]; k++) {
        int j = sorted[t.itemStart[cc] + k];
        double tr[3] = {pos[3 * (size_t)j] - t.x[3 * (size_t)cc], pos[3 * (size_t)j + 1] - t.x[3 * (size_t)cc + 1],
                        pos[3 * (size_t)j + 2] - t.x[3 * (size_t)cc + 2]};
        conv_vect(ord, tr, cv);
        for (int i = 0; i < nmo; i++) mom[(size_t)cc * NM + i] += c.h_chr[j] * cv[i];
      }
    }
  });
  for (int lev = t.depth - 1; lev >= t.height; lev--) {
    per_cube(t.levStart[lev], t.levStart[lev + 1], [&](int a, int b, double *cv) {
    for (int cc = a; cc < b; cc++) {
      int ordOut = order[cc];
      for (int k = 0; k < t.kidCount[cc]; k++) {
        int kid = t.kidStart[cc] + k, nIn = nmom(order[kid]);
        double tr[3] = {t.x[3 * (size_t)kid] - t.x[3 * (size_t)cc], t.x[3 * (size_t)kid + 1] - t.x[3 * (size_t)cc + 1],
                        t.x[3 * (size_t)kid + 2] - t.x[3 * (size_t)cc + 2]};
        conv_vect(ordOut, tr, cv);
        int nOut = nmom(ordOut);
        for (int i = 0; i < nOut; i++) {
          int i1 = mi[3 * i], i2 = mi[3 * i + 1], i3 = mi[3 * i + 2];
          double tmp = 0.0;
          for (int k1 = 0; k1 <= i1; k1++)
            for (int k2 = 0; k2 <= i2; k2++)
              for (int k3 = 0; k3 <= i3; k3++) {
                int bi = idx3[(k1 * D + k2) * D + k3];
                if (bi < nIn) tmp += cv[idx3[((i1 - k1) * D + (i2 - k2)) * D + (i3 - k3)]] * mom[(size_t)kid * NM + bi];
              }
          mom[(size_t)cc * NM + i] += tmp;
        }
      }
    }
    });
  }
  std::vector<double> spos(3 * (size_t)m), schr(m);
  for (int i = 0; i < m; i++) {
    for (int k = 0; k < 3; k++) spos[3 * (size_t)i + k] = pos[3 * (size_t)sorted[i] + k];
    schr[i] = c.h_chr[sorted[i]];
  }
  cudaStream_t s = c.stream;
  if (!d.arena.upload(&d.d_pos, spos, s) || !d.arena.upload(&d.d_chr, schr, s) ||
      !d.arena.upload(&d.d_ctr, t.x, s) || !d.arena.upload(&d.d_rad, t.rad, s) ||
      !d.arena.upload(&d.d_level, t.level, s) || !d.arena.upload(&d.d_kidStart, t.kidStart, s) ||
      !d.arena.upload(&d.d_kidCount, t.kidCount, s) || !d.arena.upload(&d.d_itemStart, t.itemStart, s) ||
      !d.arena.upload(&d.d_itemCount, t.itemCount, s) || !d.arena.upload(&d.d_order, order, s))
    return false;
  // the walks contract (-1)^|i| M_i (the sign of D^i taken at the point rather
  // than at the cube); a mixed context's walks read them in FP32
  for (size_t cc = 0; cc < (size_t)t.nCubes; cc++)
    for (int i = 0; i < NM; i++)
      if ((mi[3 * i] + mi[3 * i + 1] + mi[3 * i + 2]) & 1) mom[cc * NM + i] = -mom[cc * NM + i];
  if (c.mixed) {
    std::vector<float> smf(mom.begin(), mom.end());
    float *p = nullptr;
    if (!d.arena.upload(&p, smf, s)) return false;
    d.d_smom = p;
    FB_CUDA(cudaStreamSynchronize(s));
  } else {
    double *p = nullptr;
    if (!d.arena.upload(&p, mom, s)) return false;
    d.d_smom = p;
  }
  FB_CUDA(cudaStreamSynchronize(s));  // host vectors above are about to go out of scope
  tm.mark("charge_tree");
  d.built = true;
  return true;
}

// ---------------------------------------------------------------------------
// direct RHS: thread per panel, charges staged through shared memory
// ---------------------------------------------------------------------------
constexpr int kRhsTile = 256;

__global__ void rhs_direct_kernel(int n, int m, int q, const double *__restrict__ vtx, const double *__restrict__ nrm,
                                  const double *__restrict__ area, const double *__restrict__ pos,
                                  const double *__restrict__ chr, double fac, double *rhs) {
  __shared__ double4 sc[kRhsTile];
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = X < n;
  const int Xs = valid ? X : 0;
  const double *v0 = vtx + 9 * (size_t)Xs;
  double ax2[3], ax0[3], nx[3];
  for (int k = 0; k < 3; k++) {
    ax2[k] = v0[3 + k] - v0[k];
    ax0[k] = v0[6 + k] - v0[3 + k];
    nx[k] = nrm[3 * (size_t)Xs + k];
  }
  const double A2 = 2.0 * area[Xs];
  const double *t = c_tLeg[q], *w = c_wLeg[q];
  double s0 = 0.0, s1 = 0.0;
  for (int base = 0; base < m; base += kRhsTile) {
    const int cnt = min(kRhsTile, m - base);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x)
      sc[j] = make_double4(pos[3 * (size_t)(base + j)], pos[3 * (size_t)(base + j) + 1], pos[3 * (size_t)(base + j) + 2],
                           chr[base + j]);
    __syncthreads();
    for (int j = 0; j < cnt; j++) {
      const double4 cj = sc[j];
      const double r0[3] = {v0[0] - cj.x, v0[1] - cj.y, v0[2] - cj.z};
      double i0 = 0.0, i1 = 0.0;
      for (int ix = 0; ix < q; ix++)
        for (int jx = 0; jx < q; jx++) {
          double r[3];
          for (int k = 0; k < 3; k++) r[k] = r0[k] + t[ix] * (ax2[k] + t[jx] * ax0[k]);
          const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
          const double ri = rsqrt(r2);
          const double r3i = ri * ri * ri;
          const double ip = nx[0] * r[0] + nx[1] * r[1] + nx[2] * r[2];
          i0 += ri * t[ix] * w[ix] * w[jx];
          i1 += (-ip * r3i) * t[ix] * w[ix] * w[jx];
        }
      s0 += cj.w * (i0 * A2);
      s1 += cj.w * (i1 * A2);
    }
    __syncthreads();
  }
  if (valid) {
    rhs[X] = s0 * fac;
    rhs[n + X] = s1 * fac;
  }
}

// Mixed contexts, one-point rule (q = 1): the same direct sum in FP32.  The
// panel's quadrature point and the charges are taken relative to the root
// box centre (differences in FP64, then rounded), the pair terms use the
// MUFU reciprocal square root, and every 64 charges are summed in FP32 and
// added to the panel's FP64 totals.  The pair terms run in packed f32x2
// arithmetic (sm_100 FFMA2/FMUL2/FADD2), two charges per step.
constexpr int kRhsTileF = 1024;

__global__ void charges_to_float_kernel(int m, const double *__restrict__ pos, const double *__restrict__ chr,
                                        double ox, double oy, double oz, float4 *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  out[j] = make_float4((float)(pos[3 * (size_t)j] - ox), (float)(pos[3 * (size_t)j + 1] - oy),
                       (float)(pos[3 * (size_t)j + 2] - oz), (float)chr[j]);
}

// Stages charges [base, base + cnt) as (cnt + 1) / 2 interleaved pairs with
// negated positions, s[2p] = (-x0 -x1 -y0 -y1), s[2p + 1] = (-z0 -z1 q0 q1),
// so every packed operand is one half of a staged float4; an odd count pads
// the last pair with a copy of the last position carrying zero charge.
__device__ __forceinline__ void stage_charge_pairs(const float4 *__restrict__ chg, int base, int cnt, float4 *s) {
  for (int p = threadIdx.x; 2 * p < cnt; p += blockDim.x) {
    const float4 a = chg[base + 2 * p];
    const float4 b = 2 * p + 1 < cnt ? chg[base + 2 * p + 1] : make_float4(a.x, a.y, a.z, 0.f);
    s[2 * p] = make_float4(-a.x, -b.x, -a.y, -b.y);
    s[2 * p + 1] = make_float4(-a.z, -b.z, a.w, b.w);
  }
}

__global__ void __launch_bounds__(256)
rhs_direct_f2_kernel(int n, int m, const double *__restrict__ vtx, const double *__restrict__ nrm,
                     const double *__restrict__ area, const float4 *__restrict__ chg, double ox, double oy,
                     double oz, double fac, double *rhs) {
  __shared__ float4 sc[kRhsTileF];
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = X < n;
  const int Xs = valid ? X : 0;
  const double *v0 = vtx + 9 * (size_t)Xs;
  const double t = c_tLeg[1][0], wt = c_wLeg[1][0];
  float2 px, py, pz;
  {
    double p[3];
    for (int k = 0; k < 3; k++) p[k] = v0[k] + t * ((v0[3 + k] - v0[k]) + t * (v0[6 + k] - v0[3 + k]));
    px = f2((float)(p[0] - ox));
    py = f2((float)(p[1] - oy));
    pz = f2((float)(p[2] - oz));
  }
  const float2 nx = f2((float)nrm[3 * (size_t)Xs]), ny = f2((float)nrm[3 * (size_t)Xs + 1]),
               nz = f2((float)nrm[3 * (size_t)Xs + 2]);
  double s0 = 0.0, s1 = 0.0;
  for (int base = 0; base < m; base += kRhsTileF) {
    const int cnt = min(kRhsTileF, m - base), cnt2 = (cnt + 1) / 2;
    stage_charge_pairs(chg, base, cnt, sc);
    __syncthreads();
    for (int j0 = 0; j0 < cnt2; j0 += 32) {   // FP32 sums of 64 charges at a time
      const int j1 = min(cnt2, j0 + 32);
      float2 a0 = f2(0.f), a1 = f2(0.f);
#pragma unroll 4
      for (int j = j0; j < j1; j++) {
        const float4 A = sc[2 * j], B = sc[2 * j + 1];
        const float2 dx = __fadd2_rn(px, make_float2(A.x, A.y));
        const float2 dy = __fadd2_rn(py, make_float2(A.z, A.w));
        const float2 dz = __fadd2_rn(pz, make_float2(B.x, B.y));
        const float2 q = make_float2(B.z, B.w);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        float2 ri;
        ri.x = rsqrt_t(r2.x);
        ri.y = rsqrt_t(r2.y);
        const float2 qr3 = __fmul2_rn(q, __fmul2_rn(__fmul2_rn(ri, ri), ri));
        a0 = __ffma2_rn(q, ri, a0);
        a1 = __ffma2_rn(qr3, __ffma2_rn(nz, dz, __ffma2_rn(ny, dy, __fmul2_rn(nx, dx))), a1);
      }
      s0 += (double)a0.x + (double)a0.y;
      s1 -= (double)a1.x + (double)a1.y;
    }
    __syncthreads();
  }
  if (valid) {
    const double W = 2.0 * area[Xs] * t * wt * wt * fac;
    rhs[X] = s0 * W;
    rhs[n + X] = s1 * W;
  }
}

// ---------------------------------------------------------------------------
// charge-tree walks: mode 0 = RHS (Coulomb), 1 = energy (G0 - Gk), 2 = the
// screened term alone (the plugin ABI's energy of a reused RHS)
// ---------------------------------------------------------------------------
// A warp walks the charge tree for its 32 points (consecutive panels in tree
// order, so neighbours in space) together.  Its stack, in shared memory,
// holds (cube, lane mask) entries.  At a cube every lane of the mask makes its
// own acceptance test; the accepting lanes evaluate the cube's expansion
// together, the lanes at a leaf sum its charges, and the children are pushed
// (last child first) with the mask of the lanes that go on into them.  Each
// lane therefore visits exactly the cubes of its own depth-first walk, in the
// reference's order, while the cube records and the moments are read once per
// warp and every expansion runs at a warp-uniform order.
//
// The expansion: the derivative tensor of the radial kernel by the level
// recursion of derivs_inplace, unrolled at compile time for each order so
// that the tensor lives in registers, contracted with the signed moments
// (-1)^|i| M_i.  By linearity of the recursion in its radial sequence, the
// energy's  sum M_i D^i (G0 - Gk)  and  sum M_i n.grad D^i (eps Gk - G0)  are
// two tensors of the combined sequences (the first only to order p).  T = float
// (mixed contexts): tensors, contraction and the leaves' pair terms in FP32,
// point-to-cube offsets in FP64 and then rounded; the per-panel sums in FP64.
constexpr int kWalkThreads = 256;
constexpr int kWalkStack = 8 * 20 + 4;   // depth <= 20: at most 7 per level + 2 entries wait

struct WalkTree {
  const double *ctr, *rad, *pos, *chr;
  const int *level, *kidStart, *kidCount, *itemStart, *itemCount, *order;
  const void *smom;   // nCubes x NM signed moments, T
  double theta;
  int height, depth, NM;
};

// y0 += sum_I sm_I d_I;  g_k += sum_I sm_I d_{I + e_k}
template <bool Y0, bool Y1, int I, typename T>
__device__ __forceinline__ void contract_step(const T *__restrict__ sm, const T *d, T &y0, T &g0, T &g1, T &g2) {
  constexpr Tri m = gmi(I);
  constexpr int e1 = gidx(m.a + 1, m.b, m.c), e2 = gidx(m.a, m.b + 1, m.c), e3 = gidx(m.a, m.b, m.c + 1);
  const T s = sm[I];
  if constexpr (Y0) y0 += s * d[I];
  if constexpr (Y1) {
    g0 += s * d[e1];
    g1 += s * d[e2];
    g2 += s * d[e3];
  }
}
template <bool Y0, bool Y1, typename T, int... I>
__device__ __forceinline__ void contract(const T *__restrict__ sm, const T *d, T &y0, T &g0, T &g1, T &g2,
                                         std::integer_sequence<int, I...>) {
  (contract_step<Y0, Y1, I>(sm, d, y0, g0, g1, g2), ...);
}

// Radial sequences of derivs_inplace: G0[k] = (1/r d/dr)^k (1/(4 pi r)), and
// the screened Gk (src/kernel.c:84-104), for k <= K.
template <int K, typename T>
__device__ __forceinline__ void radial_coulomb(T r, T *G0) {
  const T r2 = (T)-1 / (r * r);
  G0[0] = (T)kFourPiI / r;
#pragma unroll
  for (int k = 0; k < K; k++) G0[k + 1] = (T)(2 * k + 1) * r2 * G0[k];
}
template <int K, typename T>
__device__ __forceinline__ void radial_screened(T r, T kappa, T *G0, T *Gk) {
  const T rexp = exp(-kappa * r), r1 = (T)1 / r, rr2 = r1 * r1, nr2 = -rr2, k2 = kappa * kappa;
  G0[0] = r1 * (T)kFourPiI;
  Gk[0] = rexp * G0[0];
  if constexpr (K >= 1) {
    G0[1] = nr2 * G0[0];
    Gk[1] = -Gk[0] * (rr2 + kappa * r1);
  }
#pragma unroll
  for (int k = 1; k < K; k++) {
    G0[k + 1] = (T)(2 * k + 1) * nr2 * G0[k];
    Gk[k + 1] = rr2 * (k2 * Gk[k - 1] - (T)(2 * k + 1) * Gk[k]);
  }
}

// The terms of one accepted cube of expansion order ORD at offset x from the
// point: y0 (potential) and y1 (normal derivative) of the walk's mode.
template <int ORD, typename T, int MODE>
__device__ __forceinline__ void cube_terms(const T *__restrict__ sm, const T *x, const T *nx, T kappa, T eps, T &y0,
                                           T &y1) {
  using Moments = std::make_integer_sequence<int, nmom_c(ORD)>;
  const T r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  T a0 = (T)0, g0 = (T)0, g1 = (T)0, g2 = (T)0;
  if constexpr (MODE == 0) {
    T G[ORD + 2], d[nmom_c(ORD + 1)];
    radial_coulomb<ORD + 1>(r, G);
    deriv_table<ORD + 1>(d, x, G);
    contract<true, true>(sm, d, a0, g0, g1, g2, Moments{});
    y0 = a0;
    y1 = nx[0] * g0 + nx[1] * g1 + nx[2] * g2;
  } else if constexpr (MODE == 1) {
    T G0[ORD + 2], Gk[ORD + 2], H[ORD + 2];
    radial_screened<ORD + 1>(r, kappa, G0, Gk);
    {
      T d[nmom_c(ORD)];
#pragma unroll
      for (int k = 0; k <= ORD; k++) H[k] = G0[k] - Gk[k];
      deriv_table<ORD>(d, x, H);
      contract<true, false>(sm, d, a0, g0, g1, g2, Moments{});
    }
    {
      T d[nmom_c(ORD + 1)];
#pragma unroll
      for (int k = 0; k <= ORD + 1; k++) H[k] = eps * Gk[k] - G0[k];
      deriv_table<ORD + 1>(d, x, H);
      contract<false, true>(sm, d, a0, g0, g1, g2, Moments{});
    }
    y0 = a0;
    y1 = nx[0] * g0 + nx[1] * g1 + nx[2] * g2;
  } else {
    T G0[ORD + 2], Gk[ORD + 2], d[nmom_c(ORD + 1)];
    radial_screened<ORD + 1>(r, kappa, G0, Gk);
    deriv_table<ORD + 1>(d, x, Gk);
    contract<true, true>(sm, d, a0, g0, g1, g2, Moments{});
    y0 = a0;
    y1 = eps * (nx[0] * g0 + nx[1] * g1 + nx[2] * g2);
  }
}

// Orders above the unrolled ones: the runtime recursion with the tensors in
// local memory.
template <int PM, typename T, int MODE>
__device__ __noinline__ void cube_terms_generic(int ord, const T *__restrict__ sm, const T *x, const T *nx, T kappa,
                                                T eps, T &y0, T &y1) {
  constexpr int ND = nmom_c(PM);
  T d0[ND], dk[ND];
  derivs_inplace<PM, T>(ord + 1, x, kappa, MODE == 0, d0, dk, 1);
  T a0 = (T)0, a1 = (T)0;
  for (int i = 0, nmo = nmom(ord); i < nmo; i++) {
    const char4 a = c_mi[i];
    const int e1 = IDX(a.x + 1, a.y, a.z), e2 = IDX(a.x, a.y + 1, a.z), e3 = IDX(a.x, a.y, a.z + 1);
    const T s = sm[i];
    if (MODE == 0) {
      a0 += s * d0[i];
      a1 += s * (nx[0] * d0[e1] + nx[1] * d0[e2] + nx[2] * d0[e3]);
    } else if (MODE == 2) {
      a0 += s * dk[i];
      a1 += s * eps * (nx[0] * dk[e1] + nx[1] * dk[e2] + nx[2] * dk[e3]);
    } else {
      a0 += s * (d0[i] - dk[i]);
      a1 += s * (eps * (nx[0] * dk[e1] + nx[1] * dk[e2] + nx[2] * dk[e3]) -
                 (nx[0] * d0[e1] + nx[1] * d0[e2] + nx[2] * d0[e3]));
    }
  }
  y0 = a0;
  y1 = a1;
}

// unrolled up to order 6 (FP32) or 5 (FP64, whose tensors take twice the registers)
template <typename T>
__host__ __device__ constexpr int walk_unroll_max() { return sizeof(T) == 4 ? 6 : 5; }

template <int ORD, int PM, typename T, int MODE>
__device__ __forceinline__ void cube_dispatch(int ord, const T *__restrict__ sm, const T *x, const T *nx, T kappa,
                                              T eps, T &y0, T &y1) {
  if constexpr (ORD < PM && ORD <= walk_unroll_max<T>()) {
    if (ord == ORD) {
      cube_terms<ORD, T, MODE>(sm, x, nx, kappa, eps, y0, y1);
      return;
    }
    cube_dispatch<ORD + 1, PM, T, MODE>(ord, sm, x, nx, kappa, eps, y0, y1);
  } else if constexpr (ORD < PM) {
    cube_terms_generic<PM, T, MODE>(ord, sm, x, nx, kappa, eps, y0, y1);
  }
}

// The walk of one point per lane; lanes with active == false only take part in
// the warp's collective steps.  y[] accumulates in the lane's visiting order.
template <int PM, typename T, int MODE>
__device__ __forceinline__ void walk_warp(const WalkTree &t, bool active, const double *qp, const T *nx, T kappa,
                                          T eps, double *y, int2 *stk) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned all = __ballot_sync(0xffffffffu, active);
  if (all == 0u) return;
  if (lane == 0) stk[0] = make_int2(0, (int)all);
  __syncwarp();
  int sp = 1;
  while (sp > 0) {
    const int2 top = stk[--sp];
    __syncwarp();   // every lane has read the entry before lane 0 may reuse its slot
    const int c = top.x;
    const unsigned mask = (unsigned)top.y;
    const bool in = (mask >> lane) & 1u;
    const double r0 = qp[0] - t.ctr[3 * (size_t)c], r1 = qp[1] - t.ctr[3 * (size_t)c + 1],
                 r2 = qp[2] - t.ctr[3 * (size_t)c + 2];
    const int lev = t.level[c];
    const bool acc = in && t.rad[c] < t.theta * sqrt(r0 * r0 + r1 * r1 + r2 * r2) && lev >= t.height;
    const unsigned accMask = __ballot_sync(0xffffffffu, acc);
    if (acc) {
      const T x[3] = {(T)r0, (T)r1, (T)r2};
      T y0 = (T)0, y1 = (T)0;
      cube_dispatch<0, PM, T, MODE>(t.order[c], static_cast<const T *>(t.smom) + (size_t)c * t.NM, x, nx, kappa,
                                    eps, y0, y1);
      if (MODE == 0) {
        y[0] += (double)y0 / kFourPiI;
        y[1] += (double)y1 / kFourPiI;
      } else {
        y[0] += (double)y0;
        y[1] += (double)y1;
      }
    }
    const unsigned rest = mask & ~accMask;
    if (rest == 0u) continue;
    if (lev == t.depth) {
      if (in && !acc) {
        for (int j = t.itemStart[c], j1 = j + t.itemCount[c]; j < j1; j++) {
          const T x[3] = {(T)(qp[0] - t.pos[3 * (size_t)j]), (T)(qp[1] - t.pos[3 * (size_t)j + 1]),
                          (T)(qp[2] - t.pos[3 * (size_t)j + 2])};
          const T rr2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
          const T ip = nx[0] * x[0] + nx[1] * x[1] + nx[2] * x[2];
          const T q = (T)t.chr[j];
          if (MODE == 0) {
            const T ri = (T)1 / sqrt(rr2), r3i = ri / rr2;
            y[0] += (double)(q * ri);
            y[1] += (double)(q * (-ip * r3i));
          } else {
            const T rn = sqrt(rr2), G0 = (T)kFourPiI / rn, ek = exp(-kappa * rn);
            const T Gk = ek * G0, coef = (kappa * rn + (T)1) * ek;
            const T dG0dn = -ip * G0 / rr2, dGkdn = coef * dG0dn;
            if (MODE == 2) {
              y[0] += (double)(q * Gk);
              y[1] += (double)(q * eps * dGkdn);
            } else {
              y[0] += (double)(q * (G0 - Gk));
              y[1] += (double)(q * (eps * dGkdn - dG0dn));
            }
          }
        }
      }
      continue;
    }
    const int k0 = t.kidStart[c], nk = t.kidCount[c];
    if (sp + nk > kWalkStack) break;   // unreachable: the host caps the depth at 20
    if (lane == 0)
      for (int k = 0; k < nk; k++) stk[sp + k] = make_int2(k0 + nk - 1 - k, (int)rest);   // first child on top
    sp += nk;
    __syncwarp();
  }
}

template <int PM, typename T, int MODE>
__global__ void __launch_bounds__(kWalkThreads)
tree_walk_kernel(int n, int q, const double *__restrict__ vtx, const double *__restrict__ nrm,
                 const double *__restrict__ area, WalkTree t, double kappa, double eps, double fac,
                 const double *__restrict__ sgm, double *rhs, double *partial) {
  __shared__ int2 stk[kWalkThreads / 32][kWalkStack];
  __shared__ double red[kWalkThreads];
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = X < n;
  const int Xs = valid ? X : 0;
  const double *v0 = vtx + 9 * (size_t)Xs;
  double ax2[3], ax0[3];
  T nx[3];
  for (int k = 0; k < 3; k++) {
    ax2[k] = v0[3 + k] - v0[k];
    ax0[k] = v0[6 + k] - v0[3 + k];
    nx[k] = (T)nrm[3 * (size_t)Xs + k];
  }
  const double *tq = c_tLeg[q], *w = c_wLeg[q];
  double o0 = 0.0, o1 = 0.0;
  for (int ix = 0; ix < q; ix++)
    for (int jx = 0; jx < q; jx++) {
      double qp[3], y[2] = {0.0, 0.0};
      for (int k = 0; k < 3; k++) qp[k] = v0[k] + tq[ix] * (ax2[k] + tq[jx] * ax0[k]);
      walk_warp<PM, T, MODE>(t, valid, qp, nx, (T)kappa, (T)eps, y, stk[threadIdx.x >> 5]);
      o0 += y[0] * tq[ix] * w[ix] * w[jx];
      o1 += y[1] * tq[ix] * w[ix] * w[jx];
    }
  double e = 0.0;
  if (valid) {
    o0 *= 2.0 * area[X];
    o1 *= 2.0 * area[X];
    if (MODE == 0) {
      rhs[X] = fac * o0;
      rhs[n + X] = fac * o1;
    } else if (MODE == 2) {
      e = -o0 * sgm[X + n] + o1 * sgm[X];   // rhsReuseEnergyWorker, treecode.c:889-910
    } else {
      e = o0 * sgm[X + n] + o1 * sgm[X];
    }
  }
  if (MODE != 0) {
    red[threadIdx.x] = e;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
  }
}

// out = sum of the k partials, in a fixed order whatever k: thread t adds
// p[t], p[t + 256], ... in turn, then a fixed shared-memory tree adds the 256
// thread sums (one block of kSumThreads threads)
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) sum_partials_kernel(int k, const double *__restrict__ p, double *out) {
  __shared__ double red[kSumThreads];
  double s = 0.0;
  for (int i = threadIdx.x; i < k; i += kSumThreads) s += p[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int m = kSumThreads / 2; m > 0; m >>= 1) {
    if ((int)threadIdx.x < m) red[threadIdx.x] += red[threadIdx.x + m];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

template <int PM>
static void launch_walk(Context &c, int mode, const double *sgm, double *rhs, double *partial) {
  ChargeTreeDev &d = *c.ct;
  // the screened-only walk uses the RHS acceptance ratio (treecode.c:731)
  const double theta = (mode == 1) ? c.prm.energy_theta : c.prm.rhs_theta;
  const WalkTree t{d.d_ctr, d.d_rad, d.d_pos, d.d_chr, d.d_level, d.d_kidStart, d.d_kidCount, d.d_itemStart,
                   d.d_itemCount, d.d_order, d.d_smom, theta, d.height, d.depth, c.NM};
  // the walks of a mixed context (RHS and energy) with FP32 cube and pair terms, FP64 sums
  auto kern = c.mixed ? (mode == 0 ? tree_walk_kernel<PM, float, 0>
                                   : mode == 1 ? tree_walk_kernel<PM, float, 1> : tree_walk_kernel<PM, float, 2>)
                      : (mode == 0 ? tree_walk_kernel<PM, double, 0>
                                   : mode == 1 ? tree_walk_kernel<PM, double, 1> : tree_walk_kernel<PM, double, 2>);
  kern<<<ceil_div(c.n, kWalkThreads), kWalkThreads, 0, c.stream>>>(
      c.n, c.prm.quad_order, c.d_vtx, c.d_nrm, c.d_area, t, c.prm.kappa, c.epsilon,
      c.rhsFac != 0.0 ? c.rhsFac : kFourPiI / c.prm.eps1, sgm, rhs, partial);
}

#define FB_DISPATCH_WALK(P, ...)                      \
  switch (P) {                                        \
    case 1: launch_walk<2>(__VA_ARGS__); break;       \
    case 2: launch_walk<3>(__VA_ARGS__); break;       \
    case 3: launch_walk<4>(__VA_ARGS__); break;       \
    case 4: launch_walk<5>(__VA_ARGS__); break;       \
    case 5: launch_walk<6>(__VA_ARGS__); break;       \
    case 6: launch_walk<7>(__VA_ARGS__); break;       \
    case 7: launch_walk<8>(__VA_ARGS__); break;       \
    default: launch_walk<9>(__VA_ARGS__); break;      \
  }

// The FP32 charge records of a mixed context (position minus the root box
// centre, charge), made on first use; the origin is returned.
bool charges_f32(Context &c, double *ox, double *oy, double *oz) {
  const bool hasRoot = c.pt.t.x.size() >= 3;
  *ox = hasRoot ? c.pt.t.x[0] : 0.0;
  *oy = hasRoot ? c.pt.t.x[1] : 0.0;
  *oz = hasRoot ? c.pt.t.x[2] : 0.0;
  if (!c.ct->d_chgF) {
    if (!c.ct->arena.alloc_n(&c.ct->d_chgF, (size_t)c.nChar)) return false;
    charges_to_float_kernel<<<ceil_div(c.nChar, 256), 256, 0, c.stream>>>(c.nChar, c.ct->d_posOrig, c.ct->d_chrOrig,
                                                                         *ox, *oy, *oz, c.ct->d_chgF);
    c.launches += 1;
    FB_CUDA(cudaGetLastError());
  }
  return true;
}

bool launch_rhs(Context &c, int useTree, double *rhs) {
  FB_CHECK(c.ct != nullptr && c.nChar > 0, "no charges set (fabipb_b200_set_charges)");
  FB_CHECK(c.prm.quad_order >= 1 && c.prm.quad_order <= 10, "quadrature order %d outside 1..10", c.prm.quad_order);
  c.launches += 1;
  if (!useTree && c.mixed && c.prm.quad_order == 1) {
    double ox, oy, oz;
    if (!charges_f32(c, &ox, &oy, &oz)) return false;
    rhs_direct_f2_kernel<<<ceil_div(c.n, 256), 256, 0, c.stream>>>(
        c.n, c.nChar, c.d_vtx, c.d_nrm, c.d_area, c.ct->d_chgF, ox, oy, oz,
        c.rhsFac != 0.0 ? c.rhsFac : kFourPiI / c.prm.eps1, rhs);
    FB_CUDA(cudaGetLastError());
    return true;
  }
  if (!useTree) {
    rhs_direct_kernel<<<ceil_div(c.n, 128), 128, 0, c.stream>>>(c.n, c.nChar, c.prm.quad_order, c.d_vtx, c.d_nrm,
                                                                c.d_area, c.ct->d_posOrig, c.ct->d_chrOrig,
                                                                c.rhsFac != 0.0 ? c.rhsFac : kFourPiI / c.prm.eps1, rhs);
    FB_CUDA(cudaGetLastError());
    return true;
  }
  if (!build_charge_tree(c)) return false;
  FB_CHECK(c.ct->depth <= 20, "charge tree depth %d above the walk stack limit", c.ct->depth);
  FB_DISPATCH_WALK(c.P, c, 0, nullptr, rhs, nullptr);
  FB_CUDA(cudaGetLastError());
  return true;
}

bool launch_energy_mode(Context &c, const double *sgm, int mode, double *raw_host) {
  FB_CHECK(c.ct != nullptr && c.nChar > 0, "no charges set (fabipb_b200_set_charges)");
  if (!build_charge_tree(c)) return false;
  ChargeTreeDev &d = *c.ct;
  const int blocks = (int)ceil_div(c.n, 256);
  if (d.partialCap < blocks + 1) {
    if (!d.arena.alloc_n(&d.d_partial, (size_t)blocks + 1)) return false;
    d.partialCap = blocks + 1;
  }
  FB_DISPATCH_WALK(c.P, c, mode, sgm, nullptr, d.d_partial);
  c.launches += 2;
  sum_partials_kernel<<<1, kSumThreads, 0, c.stream>>>(blocks, d.d_partial, d.d_partial + blocks);
  FB_CUDA(cudaGetLastError());
  FB_CUDA(cudaMemcpyAsync(raw_host, d.d_partial + blocks, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  FB_CUDA(cudaStreamSynchronize(c.stream));
  return true;
}

}  // namespace fb

namespace fb {

bool launch_energy(Context &c, const double *sgm, double *raw_host) { return launch_energy_mode(c, sgm, 1, raw_host); }

__global__ void coulomb_dot_kernel(int n, double eps1, const double *__restrict__ rhs, const double *__restrict__ sgm,
                                   double *part) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += eps1 * (rhs[i] * sgm[i + n] - rhs[i + n] * sgm[i]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// eps1 * sum_i (rhs0_i sgm1_i - rhs1_i sgm0_i)  (rhsReuseCoulombDotWorker, treecode.c:912-925)
bool abi_coulomb_dot(Context &c, const double *rhs, const double *sgm, double eps1, double *dot) {
  const int blocks = 296;
  double *part = nullptr;
  FB_CUDA(cudaMallocAsync((void **)&part, (blocks + 1) * sizeof(double), c.stream));
  coulomb_dot_kernel<<<blocks, 256, 0, c.stream>>>(c.n, eps1, rhs, sgm, part);
  sum_partials_kernel<<<1, kSumThreads, 0, c.stream>>>(blocks, part, part + blocks);
  c.launches += 2;
  cudaError_t e = cudaMemcpyAsync(dot, part + blocks, sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cudaFreeAsync(part, c.stream);
  FB_CHECK(e == cudaSuccess, "Coulomb dot failed: %s", cudaGetErrorString(e));
  return true;
}

// one-point disjoint coefficients K = Ax*Ay*KER4(mX - mY) for listed pairs;
// pairs that share a vertex are skipped (done = 0)
__global__ void disjoint_pairs_kernel(long long nPairs, const double *__restrict__ vtx, const double *__restrict__ nrm,
                                      const double *__restrict__ area, const int *__restrict__ dst,
                                      const int *__restrict__ src, double kappa, double eps, double *k) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nPairs) return;
  const int Xi = dst[t], Yi = src[t];
  PanelD X, Y;
  const double *vx = vtx + 9 * (size_t)Xi, *vy = vtx + 9 * (size_t)Yi;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) { X.v[a][b] = vx[3 * a + b]; Y.v[a][b] = vy[3 * a + b]; }
  int ix[3], iy[3];
  double *out = k + 5 * (size_t)t;
  if (common_vtx(X, Y, Xi == Yi, ix, iy) != 0) { out[4] = 0.0; return; }
  double r[3], y[4];
  for (int c = 0; c < 3; c++) {
    double mx = X.v[0][c] + 0.5 * ((X.v[1][c] - X.v[0][c]) + 0.5 * (X.v[2][c] - X.v[1][c]));
    double my = Y.v[0][c] + 0.5 * ((Y.v[1][c] - Y.v[0][c]) + 0.5 * (Y.v[2][c] - Y.v[1][c]));
    r[c] = mx - my;
  }
  ker4_d(kappa, eps, r, nrm + 3 * (size_t)Xi, nrm + 3 * (size_t)Yi, y);
  const double AA = area[Xi] * area[Yi];
  for (int i = 0; i < 4; i++) out[i] = AA * y[i];
  out[4] = 1.0;
}

bool abi_disjoint_pairs(const double *vtx, const double *nrm, const double *area, long long nPairs, const int *dst,
                        const int *src, double kappa, double eps, double *k0, double *k1, double *k2, double *k3,
                        int *done, cudaStream_t s) {
  int maxIdx = 0;
  for (long long t = 0; t < nPairs; t++) maxIdx = std::max(maxIdx, std::max(dst[t], src[t]));
  const size_t np = (size_t)maxIdx + 1;
  DevArena a;
  double *d_vtx, *d_nrm, *d_area, *d_k;
  int *d_dst, *d_src;
  bool ok = a.alloc_n(&d_vtx, 9 * np) && a.alloc_n(&d_nrm, 3 * np) && a.alloc_n(&d_area, np) &&
            a.alloc_n(&d_dst, (size_t)nPairs) && a.alloc_n(&d_src, (size_t)nPairs) && a.alloc_n(&d_k, 5 * (size_t)nPairs);
  std::vector<double> hk;
  if (ok) ok = cudaMemcpyAsync(d_vtx, vtx, 9 * np * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
               cudaMemcpyAsync(d_nrm, nrm, 3 * np * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
               cudaMemcpyAsync(d_area, area, np * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess &&
               cudaMemcpyAsync(d_dst, dst, nPairs * sizeof(int), cudaMemcpyHostToDevice, s) == cudaSuccess &&
               cudaMemcpyAsync(d_src, src, nPairs * sizeof(int), cudaMemcpyHostToDevice, s) == cudaSuccess;
  if (ok) {
    disjoint_pairs_kernel<<<ceil_div(nPairs, 256), 256, 0, s>>>(nPairs, d_vtx, d_nrm, d_area, d_dst, d_src, kappa,
                                                                eps, d_k);
    hk.resize(5 * (size_t)nPairs);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(hk.data(), d_k, hk.size() * sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
  }
  a.release();
  FB_CHECK(ok, "disjoint pair coefficients failed: %s", cudaGetErrorString(cudaGetLastError()));
  for (long long t = 0; t < nPairs; t++) {
    if (hk[5 * t + 4] == 0.0) {
      if (done) done[t] = 0;
      continue;
    }
    k0[t] = hk[5 * t]; k1[t] = hk[5 * t + 1]; k2[t] = hk[5 * t + 2]; k3[t] = hk[5 * t + 3];
    if (done) done[t] = 1;
  }
  return true;
}

}  // namespace fb
