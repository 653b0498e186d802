// fmm.cu -- Cartesian Taylor FMM passes on the device (FP64).
//
//   leaf moments/noments   src/moments.c:363-543 (calcMoments0): exact
//                          triangle moments about the leaf centre; noments are
//                          the normal-weighted ones of one order less
//   Q2M                    src/fmm.c:737-756      mom_pot = Q2M1*s_pot,
//                                                  mom_dpdn = Q2M0*s_dpdn
//   M2M                    src/expan.c:223-247, 342-382
//   M2L                    src/expan.c:138-209 (derivative tensor by the
//                          radial recurrence of src/kernel.c:84-104),
//                          src/expan.c:258-290, 471-494
//   L2L                    src/expan.c:295-326, 403-452
//   L2P                    src/fmm.c:800-831     pot = beta*pot
//                          + alpha*(Q2M0^T (lec1+lec2), Q2M1^T (lec3+lec4))
//
// Graded multi-index order (src/expan.c:39-58): within total degree n, i1
// runs 0..n and i2 0..n-i1, i3 = n-i1-i2.  All per-index tables live in
// constant memory; the convolution pair lists are built on the host once.
#include <algorithm>
#include <cmath>
#include <vector>

#include <utility>

#include "context.cuh"

namespace fb {

constexpr int kTabOrder = kMaxOrder + 2;            // derivatives to order P+1
constexpr int kTabDim = kTabOrder + 1;
constexpr int kTabN = ((kTabOrder + 1) * (kTabOrder + 2) * (kTabOrder + 3)) / 6;

__constant__ short c_idx3[kTabDim * kTabDim * kTabDim];
__constant__ char4 c_mi[kTabN];         // (i1, i2, i3, |i|)
__constant__ double c_ifact3[kTabN];
__constant__ double c_sgn3[kTabN];
__constant__ double c_fact[kTabOrder + 4];
__constant__ double c_ifact[kTabOrder + 4];

__device__ __forceinline__ int IDX(int a, int b, int c) { return c_idx3[(a * kTabDim + b) * kTabDim + c]; }

struct HostTables {
  std::vector<short> idx3;
  std::vector<char4> mi;
  std::vector<double> ifact3, sgn3, fact, ifact;
};

static HostTables make_tables() {
  HostTables h;
  h.idx3.assign(kTabDim * kTabDim * kTabDim, 0);
  int i = 0;
  for (int n = 0; n <= kTabOrder; n++)
    for (int a = 0; a <= n; a++)
      for (int b = 0; b <= n - a; b++, i++) {
        int c = n - a - b;
        h.idx3[(a * kTabDim + b) * kTabDim + c] = (short)i;
        h.mi.push_back(make_char4((char)a, (char)b, (char)c, (char)n));
      }
  h.fact.assign(kTabOrder + 4, 1.0);
  h.ifact.assign(kTabOrder + 4, 1.0);
  for (int k = 1; k < kTabOrder + 4; k++) { h.fact[k] = h.fact[k - 1] * k; h.ifact[k] = 1.0 / h.fact[k]; }
  for (size_t k = 0; k < h.mi.size(); k++) {
    char4 m = h.mi[k];
    h.ifact3.push_back(1.0 / (h.fact[m.x] * h.fact[m.y] * h.fact[m.z]));
    h.sgn3.push_back((m.w % 2) ? -1.0 : 1.0);
  }
  return h;
}

static bool upload_tables() {
  static bool done = false;
  if (done) return true;
  HostTables h = make_tables();
  FB_CUDA(cudaMemcpyToSymbol(c_idx3, h.idx3.data(), h.idx3.size() * sizeof(short)));
  FB_CUDA(cudaMemcpyToSymbol(c_mi, h.mi.data(), h.mi.size() * sizeof(char4)));
  FB_CUDA(cudaMemcpyToSymbol(c_ifact3, h.ifact3.data(), h.ifact3.size() * sizeof(double)));
  FB_CUDA(cudaMemcpyToSymbol(c_sgn3, h.sgn3.data(), h.sgn3.size() * sizeof(double)));
  FB_CUDA(cudaMemcpyToSymbol(c_fact, h.fact.data(), h.fact.size() * sizeof(double)));
  FB_CUDA(cudaMemcpyToSymbol(c_ifact, h.ifact.data(), h.ifact.size() * sizeof(double)));
  done = true;
  return true;
}

// ------------------------------------------------------------------------
// device helpers
// ------------------------------------------------------------------------

// t^g / g! for multi-index g (setupConVect, src/moments.c:390-410)
__device__ __forceinline__ double conv_entry(const double *t, int g) {
  char4 m = c_mi[g];
  double f1 = 1.0, f2 = 1.0, f3 = 1.0;
  for (int i = 0; i < m.x; i++) f1 *= t[0];
  for (int i = 0; i < m.y; i++) f2 *= t[1];
  for (int i = 0; i < m.z; i++) f3 *= t[2];
  return f1 * f2 * f3 * c_ifact3[g];
}

// D^alpha G0 and D^alpha Gk at x for |alpha| <= order (setupDerivs,
// src/expan.c:138-209).  The reference fills one table per derivative level
// p from level p+1; an entry of total degree d at level p reads only degrees
// d-1 and d-2 of level p+1, so sweeping each level from the highest degree
// down lets one table per kernel be updated in place.  Entry e of the result
// lives at d0[e*stride] (stride 1 for a private array, the block width for a
// shared-memory column).
// T = float: the same recursion in FP32 (the mixed energy walk).
template <int PM, typename T = double>
__device__ void derivs_inplace(int order, const T *x, T kappa, bool coulombOnly, T *d0, T *dk, int stride) {
  T G0[PM + 2], Gk[PM + 2];
  const T r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  if (coulombOnly) {
    const T r2 = (T)-1 / (r * r);
    G0[0] = (T)kFourPiI / r;
    for (int k = 0; k < order; k++) G0[k + 1] = (T)(2 * k + 1) * r2 * G0[k];
  } else {
    const T rexp = exp(-kappa * r), r1 = (T)1 / r, rr2 = r1 * r1, nr2 = -rr2, k2 = kappa * kappa;
    G0[0] = r1 * (T)kFourPiI;
    Gk[0] = rexp * G0[0];
    G0[1] = nr2 * G0[0];
    Gk[1] = -Gk[0] * (rr2 + kappa * r1);
    for (int k = 1; k < order; k++) {
      G0[k + 1] = (T)(2 * k + 1) * nr2 * G0[k];
      Gk[k + 1] = rr2 * (k2 * Gk[k - 1] - (T)(2 * k + 1) * Gk[k]);
    }
  }
  d0[0] = G0[order];
  if (!coulombOnly) dk[0] = Gk[order];
  for (int p = order - 1; p >= 0; p--) {
    const int rows = order - p;
    const int ne = ((rows + 1) * (rows + 2) * (rows + 3)) / 6;
    for (int e = ne - 1; e >= 1; e--) {
      const char4 m = c_mi[e];
      int a, b = -1;
      T xa, fb = (T)0;
      if (m.x >= 1) {
        a = IDX(m.x - 1, m.y, m.z); xa = x[0];
        if (m.x >= 2) { b = IDX(m.x - 2, m.y, m.z); fb = m.x - 1; }
      } else if (m.y >= 1) {
        a = IDX(0, m.y - 1, m.z); xa = x[1];
        if (m.y >= 2) { b = IDX(0, m.y - 2, m.z); fb = m.y - 1; }
      } else {
        a = IDX(0, 0, m.z - 1); xa = x[2];
        if (m.z >= 2) { b = IDX(0, 0, m.z - 2); fb = m.z - 1; }
      }
      T v0 = d0[a * stride] * xa;
      if (b >= 0) v0 += d0[b * stride] * fb;
      d0[e * stride] = v0;
      if (!coulombOnly) {
        T vk = dk[a * stride] * xa;
        if (b >= 0) vk += dk[b * stride] * fb;
        dk[e * stride] = vk;
      }
    }
    d0[0] = G0[p];
    if (!coulombOnly) dk[0] = Gk[p];
  }
}

template <int PM>
__device__ __forceinline__ void derivs(int order, const double *x, double kappa, bool coulombOnly, double *d0,
                                       double *dk) {
  derivs_inplace<PM>(order, x, kappa, coulombOnly, d0, dk, 1);
}

// ------------------------------------------------------------------------
// leaf moments (setup)
// ------------------------------------------------------------------------

// c = a (*) b over multi-indices of total degree <= order (convolution,
// src/moments.c:363-385); loops k <= alpha componentwise.
template <int PM>
__device__ void convolve_d(int order, const double *a, const double *b, double *c) {
  int nOut = ((order + 1) * (order + 2) * (order + 3)) / 6;
  for (int i = 0; i < nOut; i++) {
    char4 m = c_mi[i];
    double t = 0.0;
    for (int k1 = 0; k1 <= m.x; k1++)
      for (int k2 = 0; k2 <= m.y; k2++)
        for (int k3 = 0; k3 <= m.z; k3++) t += a[IDX(m.x - k1, m.y - k2, m.z - k3)] * b[IDX(k1, k2, k3)];
    c[i] = t;
  }
}

template <int PM>
__global__ void leaf_moments_kernel(int n, int order, const double *__restrict__ vtx, const double *__restrict__ nrm,
                                    const double *__restrict__ area, const int *__restrict__ leafOfPanel,
                                    const double *__restrict__ leafCtr, double *Q0, double *Q1) {
  constexpr int NM = nmom_c(PM);
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *v0 = vtx + 9 * (size_t)i, *v1 = v0 + 3, *v2 = v0 + 6;
  const double *nm = nrm + 3 * (size_t)i;
  const double *ctr = leafCtr + 3 * (size_t)leafOfPanel[i];
  const int nMom = ((order + 1) * (order + 2) * (order + 3)) / 6;
  double a1[3], a2[3], tr[3];
  for (int k = 0; k < 3; k++) { a1[k] = v1[k] - v0[k]; a2[k] = v2[k] - v0[k]; tr[k] = v0[k] - ctr[k]; }
  double cv1[NM], cv2[NM], buf[NM], loc[NM], tv[NM];
  double area2 = 2.0 * area[i];
  for (int e = 0; e < nMom; e++) tv[e] = conv_entry(tr, e);
  for (int job = 0; job < 2; job++) {
    int order1 = (job == 0) ? order : order - 1;
    int n1 = ((order1 + 1) * (order1 + 2) * (order1 + 3)) / 6;
    for (int e = 0; e < nMom; e++) { cv1[e] = 0.0; cv2[e] = 0.0; }
    for (int e = 0; e < n1; e++) {
      double f = c_fact[c_mi[e].w];
      cv1[e] = conv_entry(a1, e) * f;
      cv2[e] = conv_entry(a2, e) * f;
    }
    convolve_d<PM>(order, cv1, cv2, buf);
    for (int e = 0; e < nMom; e++) buf[e] *= area2 * c_ifact[c_mi[e].w + 2];
    if (job == 0) {
      for (int e = 0; e < nMom; e++) loc[e] = buf[e];
    } else {
      // calcOneNoment: Nom[alpha + e_d] += n_d * Mom[alpha] for |alpha| < order
      for (int e = 0; e < nMom; e++) loc[e] = 0.0;
      int nb = (order * (order + 1) * (order + 2)) / 6;
      for (int e = 0; e < nb; e++) {
        char4 m = c_mi[e];
        loc[IDX(m.x + 1, m.y, m.z)] += nm[0] * buf[e];
        loc[IDX(m.x, m.y + 1, m.z)] += nm[1] * buf[e];
        loc[IDX(m.x, m.y, m.z + 1)] += nm[2] * buf[e];
      }
    }
    double *Q = (job == 0) ? Q0 : Q1;
    double out[NM];
    convolve_d<PM>(order, tv, loc, out);
    for (int e = 0; e < nMom; e++) Q[(size_t)e * n + i] = out[e];
  }
}

// ------------------------------------------------------------------------
// per-matvec passes
// ------------------------------------------------------------------------

// Q2M: one block per leaf, warp w sums rows m = w, w+8, ... over the leaf panels
// swap = 1 reads the two halves of sgm exchanged (the adjoint of L2P:
// momPot <- Q1 . second half, momDpdn <- Q0 . first half).
// TQ: the leaf matrices' storage type (FP32 copies in a mixed context; the
// sums are FP64 either way)
template <typename TQ>
__global__ void q2m_kernel(int nLeaves, int n, int NMleaf, int NM, const int *__restrict__ leafStart,
                           const int *__restrict__ leafCount, const int *__restrict__ leafFmm,
                           const TQ *__restrict__ Q0, const TQ *__restrict__ Q1,
                           const double *__restrict__ sgm, int swap, double *momPot, double *momDpdn) {
  int L = blockIdx.x;
  if (L >= nLeaves) return;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int st = leafStart[L], cnt = leafCount[L], f = leafFmm[L];
  for (int m = warp; m < NMleaf; m += nw) {
    double sp = 0.0, sd = 0.0;
#pragma unroll 4
    for (int j = lane; j < cnt; j += 32) {
      sp += Q1[(size_t)m * n + st + j] * sgm[(swap ? n : 0) + st + j];
      sd += Q0[(size_t)m * n + st + j] * sgm[(swap ? 0 : n) + st + j];
    }
    for (int o = 16; o > 0; o >>= 1) {
      sp += __shfl_xor_sync(0xffffffffu, sp, o);
      sd += __shfl_xor_sync(0xffffffffu, sd, o);
    }
    if (lane == 0) {
      momPot[(size_t)f * NM + m] = sp;
      momDpdn[(size_t)f * NM + m] = sd;
    }
  }
}

// M2M: one block per parent cube at one level, one warp per child (children
// w, w + 8, ... when a cube had more than eight), lanes over the output
// coefficients; the warps' shifted moments are added in warp order.
// L2L: one warp per child cube, eight cubes per block.
constexpr int kShiftWarps = 8;

__global__ void __launch_bounds__(kShiftWarps * 32)
m2m_kernel(int first, int count, int NM, int ordOut, int ordIn, const int *__restrict__ kidFirst,
           const int *__restrict__ kidCount, const double *__restrict__ ctr, const int *__restrict__ gOff,
           const int *__restrict__ gLst, int nLst, double *momPot, double *momDpdn) {
  // per warp: shift entries a, child moments b1, b2, and the child's shifted
  // contribution o1, o2 (nOut each); then the term list (offsets, entries)
  extern __shared__ double sm[];
  if ((int)blockIdx.x >= count) return;
  const int f = first + blockIdx.x;
  const int nOut = nmom(ordOut), nIn = nmom(ordIn);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int *lstOff = reinterpret_cast<int *>(sm + (size_t)kShiftWarps * 5 * nOut), *lst = lstOff + nOut + 1;
  for (int e = threadIdx.x; e <= nOut; e += blockDim.x) lstOff[e] = gOff[e];
  for (int e = threadIdx.x; e < nLst; e += blockDim.x) lst[e] = gLst[e];
  __syncthreads();
  const int nk = kidCount[f];
  double *a = sm + (size_t)warp * 5 * nOut, *b1 = a + nOut, *b2 = b1 + nOut, *o1 = b2 + nOut, *o2 = o1 + nOut;
  for (int e = lane; e < nOut; e += 32) o1[e] = o2[e] = 0.0;
  for (int k = warp; k < nk; k += kShiftWarps) {
    const int kid = kidFirst[f] + k;
    const double t[3] = {ctr[3 * kid] - ctr[3 * f], ctr[3 * kid + 1] - ctr[3 * f + 1],
                         ctr[3 * kid + 2] - ctr[3 * f + 2]};
    __syncwarp();   // the previous child's reads of a, b1, b2 are done
    for (int e = lane; e < nOut; e += 32) {
      a[e] = conv_entry(t, e);
      b1[e] = (e < nIn) ? momPot[(size_t)kid * NM + e] : 0.0;
      b2[e] = (e < nIn) ? momDpdn[(size_t)kid * NM + e] : 0.0;
    }
    __syncwarp();
    for (int al = lane; al < nOut; al += 32) {
      double s1 = 0.0, s2 = 0.0;
      for (int q = lstOff[al]; q < lstOff[al + 1]; q++) {
        const int ent = lst[q];
        const int ia = ent & 1023, ib = (ent >> 10) & 1023;
        s1 += a[ia] * b1[ib];
        s2 += a[ia] * b2[ib];
      }
      o1[al] += s1;
      o2[al] += s2;
    }
  }
  __syncthreads();
  // the warps' contributions in warp order
  const int nw = min(nk, kShiftWarps);
  for (int al = threadIdx.x; al < nOut; al += blockDim.x) {
    double s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < nw; k++) {
      const double *ok = sm + (size_t)k * 5 * nOut + 3 * nOut;
      s1 += ok[al];
      s2 += ok[nOut + al];
    }
    momPot[(size_t)f * NM + al] = s1;
    momDpdn[(size_t)f * NM + al] = s2;
  }
}



// M2L: one block (128 threads) per destination cube with a non-empty
// interaction list, sources in batches of 64.  Threads 0..63 each build the
// derivative tensors D^a G0, D^a Gk of one source into shared-memory columns
// while threads 64..127 stage the sign-weighted source moments; then thread
// (alpha, half) accumulates the four local coefficients over half of the batch
// (convM2L: l[alpha] += sum_beta c[beta] veck[alpha+beta]), and the two halves
// are added at the end.  No atomics: every destination cube is one block.
// M2L derivative tensors depend only on the geometry (r = x_dst - x_src), so
// they are built once at setup for every interaction pair and stored
// entry-major as (D^e G0, D^e Gk) pairs, tens[e][pair], which makes the
// per-matvec loads of a warp's 32 consecutive pairs coalesced.
template <int PM>
__global__ void m2l_tensor_kernel(long long nPairs, const int *__restrict__ pairSrc, const int *__restrict__ pairDst,
                                  const double *__restrict__ ctr, const int *__restrict__ ordOfCube, double kappa,
                                  double2 *tens) {
  constexpr int NMP = nmom_c(PM);
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nPairs) return;
  const int s = pairSrc[k], f = pairDst[k];
  const int order = ordOfCube[f];
  const double r[3] = {ctr[3 * f] - ctr[3 * s], ctr[3 * f + 1] - ctr[3 * s + 1], ctr[3 * f + 2] - ctr[3 * s + 2]};
  double d0[NMP], dk[NMP];
  derivs<PM>(order, r, kappa, false, d0, dk);
  const int nm = ((order + 1) * (order + 2) * (order + 3)) / 6;
  for (int e = 0; e < NMP; e++)
    tens[(size_t)e * nPairs + k] = e < nm ? make_double2(d0[e], dk[e]) : make_double2(0.0, 0.0);
}

// Sum four values over the 32 lanes with six shuffles: after the call lane 0
// holds the total of v[0], lane 8 of v[1], lane 16 of v[2], lane 24 of v[3].
template <typename TV>
__device__ __forceinline__ TV warp_sum4(TV a, TV b, TV c, TV d, int lane) {
  const bool hi16 = lane & 16;
  TV s0 = hi16 ? a : c, s1 = hi16 ? b : d;      // sent away
  TV k0 = hi16 ? c : a, k1 = hi16 ? d : b;      // kept
  k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
  k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
  const bool hi8 = lane & 8;
  TV k = hi8 ? k1 : k0;
  k += __shfl_xor_sync(0xffffffffu, hi8 ? k0 : k1, 8);
  k += __shfl_xor_sync(0xffffffffu, k, 4);
  k += __shfl_xor_sync(0xffffffffu, k, 2);
  k += __shfl_xor_sync(0xffffffffu, k, 1);
  return k;
}

// M2L conv: one warp per destination cube.  Lanes take 32 interaction pairs
// at a time and stage their sources' sign-weighted moments in a per-lane
// shared-memory column; the warp then walks the (alpha, beta) list of the
// cube's order in lock step and, per output coefficient alpha, reduces the
// four partial sums over the lanes into a per-warp shared accumulator.
// convM2L (src/expan.c:258-290): l1 += c2*(G0-Gk), l2 += c1*(eps Gk - G0),
// l3 += c2*(G0 - Gk/eps), l4 -= c1*(G0-Gk), c = sgn3 .* moments.
template <int PM>
struct M2LShape {
  static constexpr int NMP = nmom_c(PM);
  static constexpr int W = PM <= 4 ? 4 : (PM <= 6 ? 2 : 1);   // warps per block
  static constexpr size_t warpBytes = (size_t)NMP * 32 * sizeof(double2) + 4 * NMP * sizeof(double);
  static constexpr size_t bytes = W * warpBytes;
};

//
// ADJ: the transposed interaction.  The lists are those of the transposed
// pairs (the destination is the forward source; pairIdx gives the forward
// pair whose tensor D(x_f - x_s) is used), momPot/momDpdn carry the adjoint
// local expansions (g34, g12) of the forward destinations, the sign goes with
// the output index, and the outputs are the adjoint moments
//   lec1 (pot)  += sgn (eps S2 - S1 - S3 + S4),
//   lec2 (dpdn) += sgn (S1 + S3 - S2 - S4/eps),
// with S1 = sum g12 G0, S2 = sum g12 Gk, S3 = sum g34 G0, S4 = sum g34 Gk.
template <int PM, bool ADJ>
__global__ void __launch_bounds__(M2LShape<PM>::W * 32)
m2l_kernel(int nDst, const int *__restrict__ dstList, const int *__restrict__ m2lOff,
           const int *__restrict__ m2lSrc, const int *__restrict__ pairIdx, const int *__restrict__ ordOfCube,
           const int *__restrict__ lstOff, const int *__restrict__ lst, long long nPairs,
           const double2 *__restrict__ tens, int NM, double eps, const double *__restrict__ momPot,
           const double *__restrict__ momDpdn, double *lec1, double *lec2, double *lec3, double *lec4) {
  typedef M2LShape<PM> Sh;
  constexpr int NMP = Sh::NMP;
  extern __shared__ double2 m2lSmem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sC = m2lSmem + (size_t)warp * (Sh::warpBytes / sizeof(double2));
  double *sAcc = reinterpret_cast<double *>(sC + NMP * 32);   // [4][NMP]
  const int bi = blockIdx.x * Sh::W + warp;
  if (bi >= nDst) return;  // warp-uniform
  const int f = dstList[bi];
  const int order = ordOfCube[f];
  const int nm = ((order + 1) * (order + 2) * (order + 3)) / 6;
  const int o0 = m2lOff[f], o1 = m2lOff[f + 1];
  const double ieps = 1.0 / eps;
  for (int e = lane; e < 4 * NMP; e += 32) sAcc[e] = 0.0;
  for (int b0 = o0; b0 < o1; b0 += 32) {
    const int k = b0 + lane;
    const bool live = k < o1;
    const int s = live ? m2lSrc[k] : 0;
    for (int e = 0; e < nm; e++) {
      const double sg = ADJ ? 1.0 : c_sgn3[e];
      sC[e * 32 + lane] = live ? make_double2(sg * momPot[(size_t)s * NM + e], sg * momDpdn[(size_t)s * NM + e])
                               : make_double2(0.0, 0.0);
    }
    __syncwarp();
    const double2 *T = tens + (ADJ ? pairIdx[live ? k : o0] : (live ? k : o0));
    for (int al = 0; al < nm; al++) {
      const int q0 = __ldg(lstOff + al), q1 = __ldg(lstOff + al + 1);
      const int lim = order - c_mi[al].w;
      double l1 = 0.0, l2 = 0.0, l3 = 0.0, l4 = 0.0;
#pragma unroll 4
      for (int q = q0; q < q1; q++) {
        const int ent = __ldg(lst + q);
        if ((ent >> 20) > lim) break;   // |beta| beyond this cube's order
        const int ib = ent & 1023, ig = (ent >> 10) & 1023;
        const double2 d = T[(size_t)ig * nPairs];
        const double2 c = sC[ib * 32 + lane];
        if (ADJ) {   // raw sums S1..S4
          l1 += c.y * d.x;
          l2 += c.y * d.y;
          l3 += c.x * d.x;
          l4 += c.x * d.y;
        } else {
          const double v1 = d.x - d.y;
          l1 += c.y * v1;
          l2 += c.x * (eps * d.y - d.x);
          l3 += c.y * (d.x - d.y * ieps);
          l4 -= c.x * v1;
        }
      }
      const double t = warp_sum4(l1, l2, l3, l4, lane);
      if ((lane & 7) == 0) sAcc[(lane >> 3) * NMP + al] += t;
    }
    __syncwarp();
  }
  for (int e = lane; e < nm; e += 32) {
    const size_t o = (size_t)f * NM + e;
    if (ADJ) {
      const double sg = c_sgn3[e];
      const double S1 = sAcc[e], S2 = sAcc[NMP + e], S3 = sAcc[2 * NMP + e], S4 = sAcc[3 * NMP + e];
      lec1[o] += sg * (eps * S2 - S1 - S3 + S4);
      lec2[o] += sg * (S1 + S3 - S2 - S4 * ieps);
    } else {
      lec1[o] += sAcc[e];
      lec2[o] += sAcc[NMP + e];
      lec3[o] += sAcc[2 * NMP + e];
      lec4[o] += sAcc[3 * NMP + e];
    }
  }
}

// Graded position of the multi-index (a, b, c): degree n = a+b+c first, then
// a ascending, then b ascending (the order of the expansion tables).
__host__ __device__ constexpr int gidx(int a, int b, int c) {
  return ((a + b + c) * (a + b + c + 1) * (a + b + c + 2)) / 6 + a * (a + b + c + 1) - (a * (a - 1)) / 2 + b;
}

// the multi-index at graded position i (the inverse of gidx)
struct Tri { int a, b, c; };
__host__ __device__ constexpr Tri gmi(int i) {
  for (int n = 0; n < 64; n++)
    for (int a = 0; a <= n; a++)
      for (int b = 0; b <= n - a; b++)
        if (i-- == 0) return Tri{a, b, n - a - b};
  return Tri{0, 0, 0};
}

// One step of the level recursion of derivs_inplace: kind 0 sets entry 0 to
// the radial term G[p]; kind 1 sets d[e] = d[a] x[axis] + fb d[b] (b < 0: no
// second term).
struct DerivOp { int kind, e, a, b, axis, fb, p; };
__host__ __device__ constexpr int deriv_ops(int order) {
  int s = 1;
  for (int p = order - 1; p >= 0; p--) s += nmom_c(order - p);
  return s;
}
__host__ __device__ constexpr DerivOp deriv_op(int order, int s) {
  if (s == 0) return DerivOp{0, 0, 0, -1, 0, 0, order};
  s--;
  for (int p = order - 1; p >= 0; p--) {
    for (int e = nmom_c(order - p) - 1; e >= 1; e--, s--) {
      if (s != 0) continue;
      const Tri m = gmi(e);
      if (m.a >= 1)
        return DerivOp{1, e, gidx(m.a - 1, m.b, m.c), m.a >= 2 ? gidx(m.a - 2, m.b, m.c) : -1, 0, m.a - 1, 0};
      if (m.b >= 1)
        return DerivOp{1, e, gidx(0, m.b - 1, m.c), m.b >= 2 ? gidx(0, m.b - 2, m.c) : -1, 1, m.b - 1, 0};
      return DerivOp{1, e, gidx(0, 0, m.c - 1), m.c >= 2 ? gidx(0, 0, m.c - 2) : -1, 2, m.c - 1, 0};
    }
    if (s == 0) return DerivOp{0, 0, 0, -1, 0, 0, p};
    s--;
  }
  return DerivOp{0, 0, 0, -1, 0, 0, 0};
}

template <int ORDER, int S, typename T>
__device__ __forceinline__ void deriv_step(T *d, const T *x, const T *G) {
  constexpr DerivOp op = deriv_op(ORDER, S);
  if constexpr (op.kind == 0) d[0] = G[op.p];
  else if constexpr (op.b < 0) d[op.e] = d[op.a] * x[op.axis];
  else d[op.e] = d[op.a] * x[op.axis] + d[op.b] * (T)op.fb;
}
template <int ORDER, typename T, int... S>
__device__ __forceinline__ void deriv_steps(T *d, const T *x, const T *G, std::integer_sequence<int, S...>) {
  (deriv_step<ORDER, S>(d, x, G), ...);
}
// D^e G for |e| <= ORDER from the radial sequence G[0..ORDER], into registers
template <int ORDER, typename T>
__device__ __forceinline__ void deriv_table(T *d, const T *x, const T *G) {
  deriv_steps<ORDER>(d, x, G, std::make_integer_sequence<int, deriv_ops(ORDER)>{});
}

// The same recursion on packed (D^e G0, D^e Gk) pairs in FP32 (the M2L
// tensors of a mixed context, generated in the kernel from the pair offset)
template <int ORDER, int S>
__device__ __forceinline__ void deriv_step2(float2 *d, const float2 *x, const float2 *G) {
  constexpr DerivOp op = deriv_op(ORDER, S);
  if constexpr (op.kind == 0) d[0] = G[op.p];
  else if constexpr (op.b < 0) d[op.e] = __fmul2_rn(d[op.a], x[op.axis]);
  else d[op.e] = __ffma2_rn(d[op.b], f2((float)op.fb), __fmul2_rn(d[op.a], x[op.axis]));
}
template <int ORDER, int... S>
__device__ __forceinline__ void deriv_steps2(float2 *d, const float2 *x, const float2 *G,
                                             std::integer_sequence<int, S...>) {
  (deriv_step2<ORDER, S>(d, x, G), ...);
}

// M2L conv for orders up to 5 as straight-line code: every (alpha, beta)
// entry of the convolution is a compile-time step, so each lane holds its
// pair's derivative tensors in registers (FP32: generated in the kernel from
// the pair's cube offset; FP64: loaded once per batch, all loads in flight
// together), reads its source's moments from a padded shared-memory column, and keeps the four raw sums S1 = sum c2 G0, S2 = sum c2 Gk,
// S3 = sum c1 G0, S4 = sum c1 Gk per output coefficient, with the sign
// (-1)^|beta| folded in.  The convM2L combinations (src/expan.c:258-290) are
// formed once at the end: l1 = S1 - S2, l2 = eps S4 - S3, l3 = S1 - S2/eps,
// l4 = S4 - S3.
struct M2LEntry {
  int al, ib, ig, dal, dsum, first, last;
};

// Entry q of the alpha-major (alpha, beta) list with |alpha + beta| <= PM.
template <int PM>
__host__ __device__ constexpr M2LEntry m2l_entry(int q) {
  int i = 0;
  for (int n = 0; n <= PM; n++)
    for (int a = 0; a <= n; a++)
      for (int b = 0; b <= n - a; b++) {
        const int c = n - a - b;
        for (int m = 0; m <= PM - n; m++)
          for (int a2 = 0; a2 <= m; a2++)
            for (int b2 = 0; b2 <= m - a2; b2++, i++) {
              if (i != q) continue;
              const int c2 = m - a2 - b2;
              M2LEntry e{gidx(a, b, c), gidx(a2, b2, c2), gidx(a + a2, b + b2, c + c2), n, n + m,
                         m == 0 ? 1 : 0, (m == PM - n && a2 == m) ? 1 : 0};
              return e;
            }
      }
  return M2LEntry{0, 0, 0, 0, 0, 0, 0};
}

template <int PM>
__host__ __device__ constexpr int m2l_entries() {
  int i = 0;
  for (int n = 0; n <= PM; n++) i += ((n + 1) * (n + 2) / 2) * nmom_c(PM - n);   // alphas of degree n x betas
  return i;
}

// resident blocks per SM the register allocation of m2l_unrolled_kernel aims at
#ifndef FB_M2L_MIN_BLOCKS
#define FB_M2L_MIN_BLOCKS 3
#endif
// moment staging of m2l_unrolled_kernel: flattened over (source, coefficient)
// with this many loads in flight per lane (0: one source at a time)
#ifndef FB_M2L_STAGE_FLAT
#define FB_M2L_STAGE_FLAT 1
#endif
#ifndef FB_M2L_STAGE_UNROLL
#define FB_M2L_STAGE_UNROLL 8
#endif
constexpr int kM2LStageUnroll = FB_M2L_STAGE_UNROLL;
#ifndef FB_M2L_MIN_BLOCKS_F32
#define FB_M2L_MIN_BLOCKS_F32 4
#endif

template <typename TV>
struct Vec2;
template <>
struct Vec2<double> {
  typedef double2 t;
  __device__ static double2 make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Vec2<float> {
  typedef float2 t;
  __device__ static float2 make(double a, double b) { return make_float2((float)a, (float)b); }
};

// TV: the arithmetic type of the conv (double, or float in mixed contexts);
// the per-coefficient sums across batches are always FP64.
// TSMEM (order 5 in FP64): the tensors of the batch's 32 pairs are staged in shared
// memory next to the moments instead of being held in registers.
// FP32 order-5 tensors held in registers (1: 1.39 -> 1.07 ms at 2.1M panels,
// p=5) or staged in shared memory next to the moments (0)
#ifndef FB_M2L_TREG_F32
#define FB_M2L_TREG_F32 1
#endif
// FP32 M2L tensors generated in the kernel from the cube offsets (1) or read from
// the FP32 copy of the set-up tensors (0)
#ifndef FB_M2L_GEN_F32
#define FB_M2L_GEN_F32 1
#endif
template <int PM, typename TV = double>
struct M2LUnrolledShape {
  typedef typename Vec2<TV>::t V2;
  static constexpr int NMP = nmom_c(PM);
  static constexpr bool TSMEM = PM >= 5 && !(FB_M2L_TREG_F32 && sizeof(TV) == 4);
  // FP32 tensors in registers are generated in the kernel (no tensor stream)
  static constexpr bool GEN = sizeof(TV) == 4 && !TSMEM && FB_M2L_GEN_F32;
  static constexpr int W = TSMEM ? (sizeof(TV) == 8 ? 1 : 2) : 4;   // warps per block
  static constexpr size_t colBytes = (size_t)NMP * 32 * sizeof(V2);   // moment columns (and tensor columns)
  static constexpr size_t warpBytes = (TSMEM ? 2 : 1) * colBytes + 4 * NMP * sizeof(double);   // + [4][NMP] sums
  static constexpr size_t bytes = W * warpBytes;
};

// the tensor entry ig of this lane's pair: registers or the shared column
template <int PM, typename TV, bool TSMEM>
struct M2LTensors;
template <int PM, typename TV>
struct M2LTensors<PM, TV, false> {
  typename Vec2<TV>::t v[nmom_c(PM)];
  __device__ __forceinline__ typename Vec2<TV>::t get(int ig, int) const { return v[ig]; }
};
template <int PM, typename TV>
struct M2LTensors<PM, TV, true> {
  const typename Vec2<TV>::t *col;
  __device__ __forceinline__ typename Vec2<TV>::t get(int ig, int lane) const { return col[ig * 32 + lane]; }
};

// Moment column of source j, coefficient e: XOR-swizzled so that both the
// staging stores (lanes over e) and the conv reads (lanes over j) are free of
// bank conflicts.
__device__ __forceinline__ int m2l_slot(int e, int j) { return e * 32 + (j ^ (e & 31)); }

// One (alpha, beta) entry.  FULL: the cube's order is PM, every entry counts.
// The four sums of a coefficient are reduced over the lanes (component v's
// total lands in lane 8v) and added to the warp's shared sums sAcc[v][alpha].
template <typename TV>
struct M2LSumsT {
  TV s1, s2, s3, s4;
};

// Moment readers of the conv.  M2LColMoments: the XOR-swizzled columns staged
// by plain loads.  M2LRowMoments: the lane's source row of (pot, dpdn) float2
// entries staged by bulk copies, read as float4 (entries IB, IB+1) at even IB;
// within one alpha the conv takes beta in graded order from 0, and an odd entry
// is used only if its even neighbour was (|beta| never falls), so the odd
// entry takes the upper half of the last load.
template <typename V2>
struct M2LColMoments {
  const V2 *sC;
  int lane;
  template <int IB>
  __device__ __forceinline__ V2 get() { return sC[m2l_slot(IB, lane)]; }
};
struct M2LRowMoments {
  const float2 *row;
  float4 q;
  template <int IB>
  __device__ __forceinline__ float2 get() {
    if constexpr ((IB & 1) == 0) {
      q = *reinterpret_cast<const float4 *>(row + IB);
      return make_float2(q.x, q.y);
    } else {
      return make_float2(q.z, q.w);
    }
  }
};

template <int PM, int Q, bool FULL, bool ADJ, typename TV, typename TT, typename TM>
__device__ __forceinline__ void m2l_step(M2LSumsT<TV> &S, TM &M, const TT &T, int lane, int order, double *sAcc) {
  constexpr M2LEntry E = m2l_entry<PM>(Q);
  if (E.first) S.s1 = S.s2 = S.s3 = S.s4 = (TV)0;
  if (FULL || E.dsum <= order) {
    const typename Vec2<TV>::t mo = M.template get<E.ib>();
    const typename Vec2<TV>::t d = T.get(E.ig, lane);
    if ((ADJ ? E.dal : E.dsum - E.dal) & 1) {   // (-1)^|input|, or (-1)^|output| transposed
      S.s1 -= mo.y * d.x; S.s2 -= mo.y * d.y; S.s3 -= mo.x * d.x; S.s4 -= mo.x * d.y;
    } else {
      S.s1 += mo.y * d.x; S.s2 += mo.y * d.y; S.s3 += mo.x * d.x; S.s4 += mo.x * d.y;
    }
  }
  if (E.last && (FULL || E.dal <= order)) {
    const TV t = warp_sum4<TV>(S.s1, S.s2, S.s3, S.s4, lane);
    if ((lane & 7) == 0) sAcc[(lane >> 3) * nmom_c(PM) + E.al] += (double)t;
  }
}

template <int PM, bool FULL, bool ADJ, typename TV, typename TT, typename TM, int... Q>
__device__ __forceinline__ void m2l_steps(std::integer_sequence<int, Q...>, M2LSumsT<TV> &S, TM &M, const TT &T,
                                          int lane, int order, double *sAcc) {
  (m2l_step<PM, Q, FULL, ADJ, TV, TT, TM>(S, M, T, lane, order, sAcc), ...);
}

// Lane l ends with the warp total of v[(l >> 1) & 15]: one butterfly over
// sixteen values (8 + 4 + 2 + 1 + 1 shuffles), whose first stages carry
// several independent shuffles each.
__device__ __forceinline__ float warp_sum16(const float (&v)[16], int lane) {
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4, h2 = lane & 2;
  float w[8], x[4], y[2];
#pragma unroll
  for (int i = 0; i < 8; i++)
    w[i] = (h16 ? v[i + 8] : v[i]) + __shfl_xor_sync(0xffffffffu, h16 ? v[i] : v[i + 8], 16);
#pragma unroll
  for (int i = 0; i < 4; i++)
    x[i] = (h8 ? w[i + 4] : w[i]) + __shfl_xor_sync(0xffffffffu, h8 ? w[i] : w[i + 4], 8);
#pragma unroll
  for (int i = 0; i < 2; i++)
    y[i] = (h4 ? x[i + 2] : x[i]) + __shfl_xor_sync(0xffffffffu, h4 ? x[i] : x[i + 2], 4);
  float z = (h2 ? y[1] : y[0]) + __shfl_xor_sync(0xffffffffu, h2 ? y[0] : y[1], 2);
  return z + __shfl_xor_sync(0xffffffffu, z, 1);
}

// The bulk-staged M2L's (alpha, beta) step: the conv of m2l_step (FP32), with
// the four sums of four consecutive output coefficients reduced together by
// warp_sum16 (16 shuffles for 16 sums instead of 24, and independent shuffle
// chains), lane 2j (j = 4 slot + component) adding sum j to its coefficient.
struct M2LSums16 {
  float s1, s2, s3, s4;
  float b[16];   // [slot of alpha mod 4][component]
};
template <int PM, int Q, bool FULL, bool ADJ, typename TT>
__device__ __forceinline__ void m2l_step16(M2LSums16 &S, M2LRowMoments &M, const TT &T, int lane, int order,
                                           double *sAcc) {
  constexpr M2LEntry E = m2l_entry<PM>(Q);
  if (E.first) S.s1 = S.s2 = S.s3 = S.s4 = 0.f;
  if (FULL || E.dsum <= order) {
    const float2 mo = M.template get<E.ib>();
    const float2 d = T.get(E.ig, lane);
    if ((ADJ ? E.dal : E.dsum - E.dal) & 1) {   // (-1)^|input|, or (-1)^|output| transposed
      S.s1 -= mo.y * d.x; S.s2 -= mo.y * d.y; S.s3 -= mo.x * d.x; S.s4 -= mo.x * d.y;
    } else {
      S.s1 += mo.y * d.x; S.s2 += mo.y * d.y; S.s3 += mo.x * d.x; S.s4 += mo.x * d.y;
    }
  }
  if constexpr (E.last) {
    constexpr int slot = E.al & 3;
    S.b[4 * slot] = S.s1;
    S.b[4 * slot + 1] = S.s2;
    S.b[4 * slot + 2] = S.s3;
    S.b[4 * slot + 3] = S.s4;
    if constexpr (slot == 3 || E.al == nmom_c(PM) - 1) {
      // a last group of fewer than four: the slots past E.al are reduced, not written
      const float t = warp_sum16(S.b, lane);
      const int j = (lane >> 1) & 15, al = (E.al & ~3) + (j >> 2);
      if (!(lane & 1) && al <= E.al && (FULL || c_mi[al].w <= order)) sAcc[(j & 3) * nmom_c(PM) + al] += (double)t;
    }
  }
}
template <int PM, bool FULL, bool ADJ, typename TT, int... Q>
__device__ __forceinline__ void m2l_steps16(std::integer_sequence<int, Q...>, M2LSums16 &S, M2LRowMoments &M,
                                            const TT &T, int lane, int order, double *sAcc) {
  (m2l_step16<PM, Q, FULL, ADJ, TT>(S, M, T, lane, order, sAcc), ...);
}

// The lane's FP32 M2L tensor (packed D^e G0, D^e Gk) from its pair's offset x =
// x_dst - x_src: the radial sequences of derivs_inplace, then the unrolled
// level recursion, in registers.  A lane without a pair (live false) gets the
// zero tensor.
template <int PM>
__device__ __forceinline__ void m2l_gen_tensor(const float x[3], bool live, float kappa, float2 *Tv) {
  const float r = sqrtf(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  const float rexp = expf(-kappa * r), r1 = 1.f / r, rr2 = r1 * r1, k2 = kappa * kappa;
  float2 G[PM + 1];
  G[0].x = live ? r1 * (float)kFourPiI : 0.f;
  G[0].y = rexp * G[0].x;
  if constexpr (PM >= 1) {
    G[1].x = -rr2 * G[0].x;
    G[1].y = -G[0].y * (rr2 + kappa * r1);
  }
#pragma unroll
  for (int q = 1; q < PM; q++) {
    G[q + 1].x = (float)(2 * q + 1) * -rr2 * G[q].x;
    G[q + 1].y = rr2 * (k2 * G[q - 1].y - (float)(2 * q + 1) * G[q].y);
  }
  const float2 x2[3] = {f2(x[0]), f2(x[1]), f2(x[2])};
  deriv_steps2<PM>(Tv, x2, G, std::make_integer_sequence<int, deriv_ops(PM)>{});
}

// ADJ: the transposed interaction, as for m2l_kernel.  TV = float: tensors
// (float2) and staged moments in FP32, each batch's per-coefficient sums in
// FP32, accumulated over the batches in FP64.
template <int PM, bool ADJ, typename TV>
__global__ void __launch_bounds__(M2LUnrolledShape<PM, TV>::W * 32,
                                  PM >= 5 ? 1 : (sizeof(TV) == 4 ? FB_M2L_MIN_BLOCKS_F32 : FB_M2L_MIN_BLOCKS))
m2l_unrolled_kernel(int nDst, const int *__restrict__ dstList, const int *__restrict__ m2lOff,
                    const int *__restrict__ m2lSrc, const int *__restrict__ pairIdx,
                    const int *__restrict__ ordOfCube, long long nPairs,
                    const typename Vec2<TV>::t *__restrict__ tens, const double *__restrict__ ctr, float kappa,
                    int NM, double eps, const double *__restrict__ momPot, const double *__restrict__ momDpdn,
                    double *lec1, double *lec2, double *lec3, double *lec4) {
  typedef M2LUnrolledShape<PM, TV> Sh;
  typedef typename Vec2<TV>::t V2;
  constexpr int NMP = Sh::NMP;
  extern __shared__ double2 m2luSmem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  char *wbase = reinterpret_cast<char *>(m2luSmem) + (size_t)warp * Sh::warpBytes;
  V2 *sC = reinterpret_cast<V2 *>(wbase);
  double *sAcc = reinterpret_cast<double *>(wbase + Sh::colBytes);   // [4][NMP]
  const int bi = blockIdx.x * Sh::W + warp;
  if (bi >= nDst) return;  // warp-uniform
  const int f = dstList[bi];
  const int order = ordOfCube[f];
  const int o0 = m2lOff[f], o1 = m2lOff[f + 1];
  for (int e = lane; e < 4 * NMP; e += 32) sAcc[e] = 0.0;
  for (int b0 = o0; b0 < o1; b0 += 32) {
    const int k = b0 + lane;
    const bool live = k < o1;
    const int nb = min(32, o1 - b0);
    const int mySrc = live ? m2lSrc[k] : 0;
    __syncwarp();   // the previous batch's reads of sC are done
#if FB_M2L_STAGE_FLAT
    // stage the batch's moments: the 32 x NMP (source, coefficient) entries
    // dealt over the lanes in order, so a load instruction reads consecutive
    // coefficients of one or two sources and the batch's loads are independent
#pragma unroll kM2LStageUnroll
    for (int q = lane; q < 32 * NMP; q += 32) {
      const int j = q / NMP, e = q - j * NMP;
      const int sj = __shfl_sync(0xffffffffu, mySrc, j);
      sC[m2l_slot(e, j)] = j < nb ? Vec2<TV>::make(momPot[(size_t)sj * NM + e], momDpdn[(size_t)sj * NM + e])
                                  : Vec2<TV>::make(0.0, 0.0);
    }
#else
    // stage the batch's moments: one source at a time, lanes over coefficients
#pragma unroll 1
    for (int j = 0; j < 32; j++) {
      const int sj = __shfl_sync(0xffffffffu, mySrc, j);
#pragma unroll
      for (int e0 = 0; e0 < NMP; e0 += 32) {
        const int e = e0 + lane;
        if (e < NMP)
          sC[m2l_slot(e, j)] = j < nb ? Vec2<TV>::make(momPot[(size_t)sj * NM + e], momDpdn[(size_t)sj * NM + e])
                                      : Vec2<TV>::make(0.0, 0.0);
      }
    }
#endif
    M2LTensors<PM, TV, Sh::TSMEM> T;
    if constexpr (Sh::GEN) {
      // the lane's pair tensor from its offset r = x_dst - x_src (the forward pair's cubes), by the
      // radial sequences of derivs_inplace and the unrolled level recursion, in FP32 registers
      const int dc = ADJ ? mySrc : f, sc = ADJ ? f : mySrc;
      float x[3] = {1.f, 0.f, 0.f};   // a lane past the batch: any offset (its tensor is zero)
      if (live)
        for (int q = 0; q < 3; q++) x[q] = (float)(ctr[3 * dc + q] - ctr[3 * sc + q]);
      m2l_gen_tensor<PM>(x, live, kappa, T.v);
    } else if constexpr (Sh::TSMEM) {
      const V2 *tp = tens + (ADJ ? pairIdx[live ? k : o0] : (live ? k : o0));
      V2 *sT = reinterpret_cast<V2 *>(wbase + Sh::colBytes + 4 * NMP * sizeof(double));
      for (int e = 0; e < NMP; e++) sT[e * 32 + lane] = tp[(size_t)e * nPairs];
      T.col = sT;
    } else {
      const V2 *tp = tens + (ADJ ? pairIdx[live ? k : o0] : (live ? k : o0));
#pragma unroll
      for (int e = 0; e < NMP; e++) T.v[e] = tp[(size_t)e * nPairs];
    }
    __syncwarp();
    M2LSumsT<TV> S{(TV)0, (TV)0, (TV)0, (TV)0};
    M2LColMoments<V2> M{sC, lane};
    if (order == PM)
      m2l_steps<PM, true, ADJ, TV>(std::make_integer_sequence<int, m2l_entries<PM>()>{}, S, M, T, lane, order,
                                   sAcc);
    else
      m2l_steps<PM, false, ADJ, TV>(std::make_integer_sequence<int, m2l_entries<PM>()>{}, S, M, T, lane, order,
                                    sAcc);
  }
  __syncwarp();
  const int nm = ((order + 1) * (order + 2) * (order + 3)) / 6;
  const double ieps = 1.0 / eps;
  for (int e = lane; e < nm; e += 32) {
    const double S1 = sAcc[e], S2 = sAcc[NMP + e], S3 = sAcc[2 * NMP + e], S4 = sAcc[3 * NMP + e];
    const size_t o = (size_t)f * NM + e;
    if (ADJ) {   // sign already folded in
      lec1[o] += eps * S2 - S1 - S3 + S4;
      lec2[o] += S1 + S3 - S2 - S4 * ieps;
    } else {
      lec1[o] += S1 - S2;
      lec2[o] += eps * S4 - S3;
      lec3[o] += S1 - S2 * ieps;
      lec4[o] += S4 - S3;
    }
  }
}

// ---------------------------------------------------------------------------
// M2L of mixed contexts with the moments staged by the bulk-copy (TMA) engine.
// The conv is that of m2l_unrolled_kernel<PM, ADJ, float> (generated FP32
// tensors, the same (alpha, beta) walk and sums); the staging differs:
//  * m2l_pack_kernel writes the input moments as one FP32 (pot, dpdn) row per
//    cube, NMS float2 entries (NMP rounded up to a 16-byte multiple);
//  * one warp per destination cube and per block; each lane's source row is
//    fetched with one cp.async.bulk (global -> this CTA's shared memory only) into a
//    row of the warp's buffer, completion counted on an mbarrier;
//  * two buffers: the copies of batch b+1 are in flight while batch b's
//    tensors are generated and its conv runs, so the warp waits on no moment
//    load; the next batch's source indices and cube centres are loaded one
//    batch ahead as well;
//  * shared rows of RS float2 (an odd number of 16-byte units), read as float4:
//    the 8 lanes of each quarter-warp hit distinct 16-byte bank groups.
// Every wait is bounded; a warp that gives up counts the stall in
// g_m2lStalls, waits (bounded) for its other copy in flight and writes NaN to
// its cube's local expansions, so the failure shows in the result.
// ---------------------------------------------------------------------------
__device__ unsigned int g_m2lStalls = 0;

template <int PM>
struct M2LBulkShape {
  static constexpr int NMP = nmom_c(PM);
  static constexpr int NMS = (NMP + 1) & ~1;                      // packed row: 16-byte multiple
  static constexpr int RS = ((NMS / 2) & 1) ? NMS : NMS + 2;      // shared row stride, odd in 16-byte units
  static constexpr size_t bufBytes = (size_t)32 * RS * sizeof(float2);
  static constexpr size_t accOff = 2 * bufBytes;
  static constexpr size_t barOff = accOff + 4 * NMP * sizeof(double);
  static constexpr size_t bytes = barOff + 2 * sizeof(unsigned long long);
  // resident warps per SM allowed by shared memory (1 KB reserved per block)
  static constexpr int FIT = (int)((228 * 1024) / (bytes + 1024));
  static constexpr int MINB = FIT < 1 ? 1 : (FIT > 32 ? 32 : FIT);
};

__global__ void m2l_pack_kernel(long long total, int NM, int NMS, const double *__restrict__ pot,
                                const double *__restrict__ dpdn, float2 *out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long f = i / NMS;
  const int e = (int)(i - f * NMS);
  out[i] = e < NM ? make_float2((float)pot[f * NM + e], (float)dpdn[f * NM + e]) : make_float2(0.f, 0.f);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// bounded wait for the phase of the given parity; false if it never completed
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  const unsigned a = smem_u32(bar);
  for (int i = 0; i < (1 << 22); i++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// one bulk copy global -> this CTA's shared memory, counted on bar
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// the copies of the batch starting at b (nb sources, lane j's source sj) into buf
template <int PM>
__device__ __forceinline__ void m2l_bulk_issue(int nb, int sj, int lane, const float2 *__restrict__ momF, float2 *buf,
                                               unsigned long long *bar) {
  typedef M2LBulkShape<PM> Sh;
  __syncwarp();
  // the generic-proxy reads of this buffer (the conv two batches back) are
  // ordered before the async-proxy writes that follow
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (lane == 0) mbar_expect_tx(bar, (unsigned)(nb * Sh::NMS * sizeof(float2)));
  __syncwarp();
  if (lane < nb) bulk_g2s(buf + lane * Sh::RS, momF + (size_t)sj * Sh::NMS, Sh::NMS * sizeof(float2), bar);
}

template <int PM, bool ADJ>
__global__ void __launch_bounds__(32, M2LBulkShape<PM>::MINB)
m2l_bulk_kernel(const int *__restrict__ dstList, const int *__restrict__ m2lOff, const int *__restrict__ m2lSrc,
                const int *__restrict__ ordOfCube, const double *__restrict__ ctr, float kappa, int NM, double eps,
                const float2 *__restrict__ momF, double *lec1, double *lec2, double *lec3, double *lec4) {
  typedef M2LBulkShape<PM> Sh;
  constexpr int NMP = Sh::NMP;
  extern __shared__ __align__(16) unsigned char m2lbSmem[];
  float2 *buf = reinterpret_cast<float2 *>(m2lbSmem);   // [2][32][RS]
  double *sAcc = reinterpret_cast<double *>(m2lbSmem + Sh::accOff);   // [4][NMP]
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(m2lbSmem + Sh::barOff);
  const int lane = threadIdx.x;
  const int f = dstList[blockIdx.x];
  const int order = ordOfCube[f];
  const int o0 = m2lOff[f], o1 = m2lOff[f + 1];
  for (int e = lane; e < 4 * NMP; e += 32) sAcc[e] = 0.0;
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const double cf0 = ctr[3 * f], cf1 = ctr[3 * f + 1], cf2 = ctr[3 * f + 2];
  // batch 0 in flight; batch 1's sources and batch 0's centres loaded
  int srcCur = o0 + lane < o1 ? m2lSrc[o0 + lane] : 0;
  m2l_bulk_issue<PM>(min(32, o1 - o0), srcCur, lane, momF, buf, &bar[0]);
  int srcNext = o0 + 32 + lane < o1 ? m2lSrc[o0 + 32 + lane] : 0;
  double cs0 = ctr[3 * srcCur], cs1 = ctr[3 * srcCur + 1], cs2 = ctr[3 * srcCur + 2];
  unsigned phase = 0;   // bit s: the parity to wait for on bar[s]
  bool bad = false;
  int it = 0;
  for (int b0 = o0; b0 < o1; b0 += 32, it++) {
    const int s = it & 1;
    const bool live = b0 + lane < o1;
    const bool more = b0 + 32 < o1;
    if (more) m2l_bulk_issue<PM>(min(32, o1 - b0 - 32), srcNext, lane, momF, buf + (s ^ 1) * 32 * Sh::RS, &bar[s ^ 1]);
    const int srcNext2 = b0 + 64 + lane < o1 ? m2lSrc[b0 + 64 + lane] : 0;
    const double cn0 = ctr[3 * srcNext], cn1 = ctr[3 * srcNext + 1], cn2 = ctr[3 * srcNext + 2];
    // the lane's tensor from the pair's offset (forward: x_dst - x_src; transposed: the
    // forward pair's cubes, x_src - x_dst here)
    M2LTensors<PM, float, false> T;
    {
      float x[3] = {1.f, 0.f, 0.f};
      if (live) {
        if (ADJ) {
          x[0] = (float)(cs0 - cf0); x[1] = (float)(cs1 - cf1); x[2] = (float)(cs2 - cf2);
        } else {
          x[0] = (float)(cf0 - cs0); x[1] = (float)(cf1 - cs1); x[2] = (float)(cf2 - cs2);
        }
      }
      m2l_gen_tensor<PM>(x, live, kappa, T.v);
    }
    const bool ok = mbar_wait(&bar[s], (phase >> s) & 1);
    phase ^= 1u << s;
    if (!__all_sync(0xffffffffu, ok)) {
      bad = true;
      if (more) mbar_wait(&bar[s ^ 1], (phase >> (s ^ 1)) & 1);
      break;
    }
    // a lane past the batch reads row 0 (finite moments) with its zero tensor
    M2LRowMoments M{buf + s * 32 * Sh::RS + (live ? lane : 0) * Sh::RS, make_float4(0.f, 0.f, 0.f, 0.f)};
    M2LSums16 S{};
    if (order == PM)
      m2l_steps16<PM, true, ADJ>(std::make_integer_sequence<int, m2l_entries<PM>()>{}, S, M, T, lane, order, sAcc);
    else
      m2l_steps16<PM, false, ADJ>(std::make_integer_sequence<int, m2l_entries<PM>()>{}, S, M, T, lane, order, sAcc);
    srcNext = srcNext2;
    cs0 = cn0; cs1 = cn1; cs2 = cn2;
  }
  __syncwarp();
  const int nm = ((order + 1) * (order + 2) * (order + 3)) / 6;
  if (bad) {
    if (lane == 0) atomicAdd(&g_m2lStalls, 1u);
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    for (int e = lane; e < nm; e += 32) {
      const size_t o = (size_t)f * NM + e;
      lec1[o] = nan;
      lec2[o] = nan;
      if (!ADJ) {
        lec3[o] = nan;
        lec4[o] = nan;
      }
    }
    return;
  }
  const double ieps = 1.0 / eps;
  for (int e = lane; e < nm; e += 32) {
    const double S1 = sAcc[e], S2 = sAcc[NMP + e], S3 = sAcc[2 * NMP + e], S4 = sAcc[3 * NMP + e];
    const size_t o = (size_t)f * NM + e;
    if (ADJ) {   // sign already folded in
      lec1[o] += eps * S2 - S1 - S3 + S4;
      lec2[o] += S1 + S3 - S2 - S4 * ieps;
    } else {
      lec1[o] += S1 - S2;
      lec2[o] += eps * S4 - S3;
      lec3[o] += S1 - S2 * ieps;
      lec4[o] += S4 - S3;
    }
  }
}

__global__ void tensors_to_float_kernel(long long n, const double2 *__restrict__ a, float2 *b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}

__global__ void to_float_kernel(long long n, const double *__restrict__ a, float *b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// L2L: one warp per child cube of one level (parents one level up)
__global__ void __launch_bounds__(kShiftWarps * 32)
l2l_kernel(int first, int count, int NM, int ordIn, int ordOut, const int *__restrict__ parent,
           const double *__restrict__ ctr, const int *__restrict__ gOff, const int *__restrict__ gLst, int nLst,
           double *lec1, double *lec2, double *lec3, double *lec4) {
  // per warp: shift entries a and the parent's locals i1..i4 (nIn each); then
  // the term list (offsets, entries)
  extern __shared__ double sm[];
  const int nIn = nmom(ordIn), nOut = nmom(ordOut);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int *lstOff = reinterpret_cast<int *>(sm + (size_t)kShiftWarps * 5 * nIn), *lst = lstOff + nOut + 1;
  for (int e = threadIdx.x; e <= nOut; e += blockDim.x) lstOff[e] = gOff[e];
  for (int e = threadIdx.x; e < nLst; e += blockDim.x) lst[e] = gLst[e];
  __syncthreads();
  const int cube = blockIdx.x * kShiftWarps + warp;
  if (cube >= count) return;   // warp-uniform; no block barrier follows
  double *a = sm + (size_t)warp * 5 * nIn, *i1 = a + nIn, *i2 = i1 + nIn, *i3 = i2 + nIn, *i4 = i3 + nIn;
  const int f = first + cube;
  const int p = parent[f];
  const double t[3] = {ctr[3 * f] - ctr[3 * p], ctr[3 * f + 1] - ctr[3 * p + 1], ctr[3 * f + 2] - ctr[3 * p + 2]};
  for (int e = lane; e < nIn; e += 32) {
    a[e] = conv_entry(t, e);
    i1[e] = lec1[(size_t)p * NM + e];
    i2[e] = lec2[(size_t)p * NM + e];
    i3[e] = lec3[(size_t)p * NM + e];
    i4[e] = lec4[(size_t)p * NM + e];
  }
  __syncwarp();
  for (int al = lane; al < nOut; al += 32) {
    const int degA = c_mi[al].w;
    double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
    for (int q = lstOff[al]; q < lstOff[al + 1]; q++) {
      const int ent = lst[q];
      const int ib = ent & 1023, ig = (ent >> 10) & 1023, db = ent >> 20;
      if (db > ordIn - degA) break;
      t1 += a[ib] * i1[ig];
      t2 += a[ib] * i2[ig];
      t3 += a[ib] * i3[ig];
      t4 += a[ib] * i4[ig];
    }
    lec1[(size_t)f * NM + al] += t1;
    lec2[(size_t)f * NM + al] += t2;
    lec3[(size_t)f * NM + al] += t3;
    lec4[(size_t)f * NM + al] += t4;
  }
}

// L2P: out[i] = beta*out[i] + alpha*Q0^T(lec1+lec2) + s1*A*x[i]  (and the
// dpdn half with Q1, lec3+lec4, s2).  diagX may be null.
template <typename TQ>
__global__ void l2p_kernel(int n, int NMleaf, int NM, const int *__restrict__ leafOfPanel,
                           const int *__restrict__ leafFmm, const TQ *__restrict__ Q0,
                           const TQ *__restrict__ Q1, const double *__restrict__ lec1,
                           const double *__restrict__ lec2, const double *__restrict__ lec3,
                           const double *__restrict__ lec4, double alpha, double beta, const double *__restrict__ area,
                           const double *__restrict__ diagX, double s1, double s2, int swap,
                           const double *__restrict__ addend, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t f = (size_t)leafFmm[leafOfPanel[i]] * NM;
  double a = 0.0, b = 0.0;
  for (int m = 0; m < NMleaf; m++) {
    a += (double)Q0[(size_t)m * n + i] * (lec1[f + m] + lec2[f + m]);
    b += (double)Q1[(size_t)m * n + i] * (lec3[f + m] + lec4[f + m]);
  }
  if (swap) {   // the adjoint of Q2M: the Q0 value belongs to the dpdn half
    const double t = a;
    a = b;
    b = t;
  }
  double o0 = (beta == 0.0) ? 0.0 : beta * out[i];
  double o1 = (beta == 0.0) ? 0.0 : beta * out[n + i];
  o0 += alpha * a;
  o1 += alpha * b;
  if (diagX) {
    o0 += s1 * area[i] * diagX[i];
    o1 += s2 * area[i] * diagX[n + i];
  }
  if (addend) {
    o0 += addend[i];
    o1 += addend[n + i];
  }
  out[i] = o0;
  out[n + i] = o1;
}

// ------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------


template <int PM>
static void launch_leaf_moments(Context &c, int order) {
  leaf_moments_kernel<PM><<<ceil_div(c.n, 64), 64, 0, c.stream>>>(c.n, order, c.d_vtx, c.d_nrm, c.d_area,
                                                                   c.d_leafOfPanel, c.d_leafCtr, c.d_Q0, c.d_Q1);
}

// Forward: moments (d_mom) -> local expansions (4 planes of d_lec).
// Adjoint: adjoint locals g12, g34 (planes 0, 1 of d_lec) -> adjoint moments
// (pot, dpdn: planes 0, 1 of d_mom) over the transposed pair lists.
template <int PU, bool ADJ, typename TV>
static void launch_m2l_unrolled(Context &c, int nDst, const int *dst, const int *off, const int *src,
                                const int *pairIdx, const void *tens, const double *inPot, const double *inDpdn,
                                double *o1, double *o2, double *o3, double *o4) {
  typedef M2LUnrolledShape<PU, TV> Sh;
  static bool attrDone = false;
  if (!attrDone) {
    cudaFuncSetAttribute(m2l_unrolled_kernel<PU, ADJ, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Sh::bytes);
    attrDone = true;
  }
  const unsigned grid = ceil_div((long long)nDst, Sh::W);
  m2l_unrolled_kernel<PU, ADJ, TV><<<grid, Sh::W * 32, Sh::bytes, c.stream>>>(
      nDst, dst, off, src, pairIdx, c.d_ordM2L, c.nM2LPairs, (const typename Vec2<TV>::t *)tens, c.d_cubeCtr,
      (float)c.prm.kappa, c.NM, c.epsilon, inPot, inDpdn, o1, o2, o3, o4);
}

// The bulk-copy staged M2L of a mixed context: the input rows packed to FP32,
// then one warp per destination cube.
template <int PU, bool ADJ>
static void launch_m2l_bulk(Context &c, int nDst, const int *dst, const int *off, const int *src,
                            const double *inPot, const double *inDpdn, double *o1, double *o2, double *o3,
                            double *o4) {
  typedef M2LBulkShape<PU> Sh;
  static bool attrDone = false;
  if (!attrDone) {
    cudaFuncSetAttribute(m2l_bulk_kernel<PU, ADJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::bytes);
    attrDone = true;
  }
  const long long total = (long long)c.pt.nFmm * Sh::NMS;
  m2l_pack_kernel<<<ceil_div(total, 256), 256, 0, c.stream>>>(total, c.NM, Sh::NMS, inPot, inDpdn, c.d_momF2);
  m2l_bulk_kernel<PU, ADJ><<<nDst, 32, Sh::bytes, c.stream>>>(dst, off, src, c.d_ordM2L, c.d_cubeCtr,
                                                              (float)c.prm.kappa, c.NM, c.epsilon, c.d_momF2, o1,
                                                              o2, o3, o4);
  c.launches += 1;   // the pack
}

// Forward: moments (d_mom) -> local expansions (4 planes of d_lec).
// Adjoint: adjoint locals g12, g34 (planes 0, 1 of d_lec) -> adjoint moments
// (pot, dpdn: planes 0, 1 of d_mom) over the transposed pair lists.
// fp32: the FP32 conv of a mixed context (orders up to 5).
template <int PM>
static void launch_m2l_t(Context &c, bool adj, bool fp32) {
  const size_t plane = (size_t)c.pt.nFmm * c.NM;
  const int nDst = adj ? (int)c.h_m2lDstT.size() : (int)c.h_m2lDst.size();
  const int *dst = adj ? c.d_m2lDstT : c.d_m2lDst, *off = adj ? c.d_m2lOffT : c.d_m2lOff;
  const int *src = adj ? c.d_m2lSrcT : c.d_m2lSrc, *pairIdx = adj ? c.d_m2lPairT : nullptr;
  const double *inPot = adj ? c.d_lec + plane : c.d_mom, *inDpdn = adj ? c.d_lec : c.d_mom + plane;
  double *o1 = adj ? c.d_mom : c.d_lec, *o2 = adj ? c.d_mom + plane : c.d_lec + plane;
  double *o3 = c.d_lec + 2 * plane, *o4 = c.d_lec + 3 * plane;
  if (PM <= 5) {
    constexpr int PU = PM <= 5 ? PM : 5;
    if (fp32 && c.d_momF2) {
      if (adj) launch_m2l_bulk<PU, true>(c, nDst, dst, off, src, inPot, inDpdn, o1, o2, o3, o4);
      else launch_m2l_bulk<PU, false>(c, nDst, dst, off, src, inPot, inDpdn, o1, o2, o3, o4);
    } else if (fp32 && (M2LUnrolledShape<PU, float>::GEN || c.d_m2lTensF)) {
      if (adj) launch_m2l_unrolled<PU, true, float>(c, nDst, dst, off, src, pairIdx, c.d_m2lTensF, inPot, inDpdn, o1, o2, o3, o4);
      else launch_m2l_unrolled<PU, false, float>(c, nDst, dst, off, src, pairIdx, c.d_m2lTensF, inPot, inDpdn, o1, o2, o3, o4);
    } else {
      if (adj) launch_m2l_unrolled<PU, true, double>(c, nDst, dst, off, src, pairIdx, c.d_m2lTens, inPot, inDpdn, o1, o2, o3, o4);
      else launch_m2l_unrolled<PU, false, double>(c, nDst, dst, off, src, pairIdx, c.d_m2lTens, inPot, inDpdn, o1, o2, o3, o4);
    }
    return;
  }
  typedef M2LShape<PM> Sh;
  static int attrDone[2] = {0, 0};
  if (!attrDone[adj]) {
    cudaFuncSetAttribute(adj ? m2l_kernel<PM, true> : m2l_kernel<PM, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::bytes);
    attrDone[adj] = 1;
  }
  const unsigned grid = ceil_div((long long)nDst, Sh::W);
  if (adj)
    m2l_kernel<PM, true><<<grid, Sh::W * 32, Sh::bytes, c.stream>>>(nDst, dst, off, src, pairIdx, c.d_ordM2L,
                                                                    c.d_lstOff, c.d_lst, c.nM2LPairs, c.d_m2lTens,
                                                                    c.NM, c.epsilon, inPot, inDpdn, o1, o2, o3, o4);
  else
    m2l_kernel<PM, false><<<grid, Sh::W * 32, Sh::bytes, c.stream>>>(nDst, dst, off, src, pairIdx, c.d_ordM2L,
                                                                     c.d_lstOff, c.d_lst, c.nM2LPairs, c.d_m2lTens,
                                                                     c.NM, c.epsilon, inPot, inDpdn, o1, o2, o3, o4);
}

template <int PM>
static void launch_m2l_tensors(Context &c, const int *d_pairDst) {
  m2l_tensor_kernel<PM><<<ceil_div(c.nM2LPairs, 128), 128, 0, c.stream>>>(c.nM2LPairs, c.d_m2lSrc, d_pairDst,
                                                                         c.d_cubeCtr, c.d_ordM2L, c.prm.kappa,
                                                                         c.d_m2lTens);
}

#define FB_DISPATCH_ORDER(P, FN, ...)        \
  switch (P) {                               \
    case 1: FN<1>(__VA_ARGS__); break;       \
    case 2: FN<2>(__VA_ARGS__); break;       \
    case 3: FN<3>(__VA_ARGS__); break;       \
    case 4: FN<4>(__VA_ARGS__); break;       \
    case 5: FN<5>(__VA_ARGS__); break;       \
    case 6: FN<6>(__VA_ARGS__); break;       \
    case 7: FN<7>(__VA_ARGS__); break;       \
    default: FN<8>(__VA_ARGS__); break;      \
  }

bool setup_fmm(Context &c) {
  if (!upload_tables()) return false;
  const PanelTree &pt = c.pt;
  const Octree &t = pt.t;
  cudaStream_t s = c.stream;
  c.P = pt.maxOrder;
  c.NM = nmom(c.P);
  c.leafOrder = pt.ordMom[t.depth];
  c.NMleaf = nmom(c.leafOrder);
  FB_CHECK(c.P >= 0 && c.P <= kMaxOrder, "order %d outside 0..%d", c.P, kMaxOrder);

  // convolution lists for orders up to P
  std::vector<int> lstOff(c.NM + 1, 0), lst, mOff(c.NM + 1, 0), mLst;
  HostTables h = make_tables();
  auto idx = [&](int a, int b, int cc) { return (int)h.idx3[(a * kTabDim + b) * kTabDim + cc]; };
  for (int al = 0; al < c.NM; al++) {
    char4 m = h.mi[al];
    lstOff[al] = (int)lst.size();
    // beta in graded order (the j loop of convM2L/convL2L)
    for (int j = 0; j < c.NM; j++) {
      char4 b = h.mi[j];
      if (m.w + b.w > c.P) break;
      lst.push_back(j | (idx(m.x + b.x, m.y + b.y, m.z + b.z) << 10) | ((int)b.w << 20));
    }
    mOff[al] = (int)mLst.size();
    for (int k1 = 0; k1 <= m.x; k1++)
      for (int k2 = 0; k2 <= m.y; k2++)
        for (int k3 = 0; k3 <= m.z; k3++) mLst.push_back(idx(m.x - k1, m.y - k2, m.z - k3) | (idx(k1, k2, k3) << 10));
  }
  lstOff[c.NM] = (int)lst.size();
  mOff[c.NM] = (int)mLst.size();
  c.nConvList = (int)lst.size();
  c.h_lstOff = lstOff;
  c.h_mOff = mOff;
  if (!c.arena.upload(&c.d_lstOff, lstOff, s) || !c.arena.upload(&c.d_lst, lst, s) ||
      !c.arena.upload(&c.d_mOff, mOff, s) || !c.arena.upload(&c.d_mLst, mLst, s))
    return false;

  // cube data in FMM order
  std::vector<double> ctr(3 * (size_t)pt.nFmm);
  std::vector<int> parent(pt.nFmm, -1), kidFirst(pt.nFmm, 0), kidCount(pt.nFmm, 0), ordM2L(pt.nFmm);
  for (int f = 0; f < pt.nFmm; f++) {
    int cc = pt.fmmCube[f];
    for (int k = 0; k < 3; k++) ctr[3 * (size_t)f + k] = t.x[3 * (size_t)cc + k];
    ordM2L[f] = pt.ordM2L[t.level[cc]];
    if (t.level[cc] > t.height) parent[f] = pt.cubeFmm[t.parent[cc]];
    if (t.level[cc] < t.depth) {
      kidFirst[f] = pt.cubeFmm[t.kidStart[cc]];
      kidCount[f] = t.kidCount[cc];
    }
  }
  std::vector<int> leafFmm(pt.nLeaves);
  for (int L = 0; L < pt.nLeaves; L++) leafFmm[L] = pt.cubeFmm[pt.leafCube[L]];
  c.h_m2lDst.clear();
  for (int f = 0; f < pt.nFmm; f++)
    if (pt.m2lOff[f + 1] > pt.m2lOff[f]) c.h_m2lDst.push_back(f);
  if (!c.arena.upload(&c.d_cubeCtr, ctr, s) || !c.arena.upload(&c.d_fmmParent, parent, s) ||
      !c.arena.upload(&c.d_kidFirst, kidFirst, s) || !c.arena.upload(&c.d_kidCount, kidCount, s) ||
      !c.arena.upload(&c.d_ordM2L, ordM2L, s) || !c.arena.upload(&c.d_leafFmm, leafFmm, s) ||
      !c.arena.upload(&c.d_m2lOff, pt.m2lOff, s) || !c.arena.upload(&c.d_m2lSrc, pt.m2lSrc, s) ||
      !c.arena.upload(&c.d_m2lDst, c.h_m2lDst, s))
    return false;
  if (!c.arena.alloc_n(&c.d_mom, 2 * (size_t)pt.nFmm * c.NM) || !c.arena.alloc_n(&c.d_lec, 4 * (size_t)pt.nFmm * c.NM))
    return false;
  StageTimer tm("fmm_setup", s);
  // M2L derivative tensors, once per geometry
  c.nM2LPairs = (long long)pt.m2lSrc.size();
  if (c.nM2LPairs > 0) {
    std::vector<int> pairDst(pt.m2lSrc.size());
    for (int f = 0; f < pt.nFmm; f++)
      for (int k = pt.m2lOff[f]; k < pt.m2lOff[f + 1]; k++) pairDst[k] = f;
    int *d_pairDst = nullptr;
    if (!c.arena.upload(&d_pairDst, pairDst, s)) return false;
    if (!c.arena.alloc_n(&c.d_m2lTens, (size_t)c.NM * c.nM2LPairs)) return false;
    FB_DISPATCH_ORDER(c.P, launch_m2l_tensors, c, d_pairDst);
    FB_CUDA(cudaGetLastError());
    const bool genF32 = c.P == 5 ? M2LUnrolledShape<5, float>::GEN : M2LUnrolledShape<4, float>::GEN;
    if (c.mixed && c.P <= 5 && !genF32) {   // the FP32 copy the mixed conv reads
      if (!c.arena.alloc_n(&c.d_m2lTensF, (size_t)c.NM * c.nM2LPairs)) return false;
      tensors_to_float_kernel<<<1184, 256, 0, s>>>((long long)c.NM * c.nM2LPairs, c.d_m2lTens, c.d_m2lTensF);
      FB_CUDA(cudaGetLastError());
    }
    // the FP32 rows the bulk-copy staged M2L reads; FABIPB_B200_M2L_BULK=0 at
    // context creation keeps the plain-load staging (m2l_unrolled_kernel)
    const char *bulkEnv = getenv("FABIPB_B200_M2L_BULK");
    if (c.mixed && c.P <= 5 && genF32 && !(bulkEnv && atoi(bulkEnv) == 0)) {
      c.momF2Stride = (c.NM + 1) & ~1;
      if (!c.arena.alloc_n(&c.d_momF2, (size_t)pt.nFmm * c.momF2Stride)) return false;
    }
  }
  // leaf matrices
  if (!c.arena.alloc_n(&c.d_Q0, (size_t)c.NMleaf * c.n) || !c.arena.alloc_n(&c.d_Q1, (size_t)c.NMleaf * c.n))
    return false;
  FB_CHECK(c.leafOrder >= 1, "leaf moment order %d must be >= 1", c.leafOrder);
  tm.mark("m2l_tensors");
  FB_DISPATCH_ORDER(c.leafOrder, launch_leaf_moments, c, c.leafOrder);
  FB_CUDA(cudaGetLastError());
  if (c.mixed) {   // the FP32 copies Q2M and L2P read in a mixed context
    const long long nq = (long long)c.NMleaf * c.n;
    if (!c.arena.alloc_n(&c.d_Q0F, (size_t)nq) || !c.arena.alloc_n(&c.d_Q1F, (size_t)nq)) return false;
    to_float_kernel<<<1184, 256, 0, s>>>(nq, c.d_Q0, c.d_Q0F);
    to_float_kernel<<<1184, 256, 0, s>>>(nq, c.d_Q1, c.d_Q1F);
    FB_CUDA(cudaGetLastError());
  }
  tm.mark("leaf_moments");
  return true;
}

// Transposed M2L lists (built at context set-up): for every cube s
// the forward pairs (f <- s) as entries (source f, forward pair index), f
// ascending.
static bool setup_m2l_adjoint(Context &c) {
  if (c.m2lAdjReady) return true;
  const PanelTree &pt = c.pt;
  std::vector<int> offT(pt.nFmm + 1, 0), srcT(pt.m2lSrc.size()), pairT(pt.m2lSrc.size());
  for (size_t k = 0; k < pt.m2lSrc.size(); k++) offT[pt.m2lSrc[k] + 1]++;
  for (int f = 0; f < pt.nFmm; f++) offT[f + 1] += offT[f];
  std::vector<int> cur(offT.begin(), offT.end() - 1);
  for (int f = 0; f < pt.nFmm; f++)   // f ascending within each transposed list
    for (int k = pt.m2lOff[f]; k < pt.m2lOff[f + 1]; k++) {
      const int sidx = pt.m2lSrc[k];
      srcT[cur[sidx]] = f;
      pairT[cur[sidx]++] = k;
    }
  c.h_m2lDstT.clear();
  for (int f = 0; f < pt.nFmm; f++)
    if (offT[f + 1] > offT[f]) c.h_m2lDstT.push_back(f);
  if (!c.arena.upload(&c.d_m2lOffT, offT, c.stream) || !c.arena.upload(&c.d_m2lSrcT, srcT, c.stream) ||
      !c.arena.upload(&c.d_m2lPairT, pairT, c.stream) || !c.arena.upload(&c.d_m2lDstT, c.h_m2lDstT, c.stream))
    return false;
  c.m2lAdjReady = true;
  return true;
}

// Forward: Q2M, M2M, M2L, L2L; the leaves' local expansions end in d_lec.
// Adjoint (the transposed far operator, read right to left): L2P^T (Q2M with
// the halves exchanged) -> g12, g34 in d_lec planes 0, 1; L2L^T, which is the
// M2M shift; M2L^T into d_mom planes 0, 1 (adjoint moments pot, dpdn); M2M^T,
// which is the L2L shift; launch_l2p(adjoint) then applies Q2M^T.
bool launch_far_upward(Context &c, const double *sgm, bool adjoint, cudaEvent_t *marks, bool fp64) {
  const PanelTree &pt = c.pt;
  const int depth = pt.t.depth, height = pt.t.height;
  cudaStream_t s = c.stream;
  const size_t plane = (size_t)pt.nFmm * c.NM;
  if (adjoint && !setup_m2l_adjoint(c)) return false;
  FB_CUDA(cudaMemsetAsync(c.d_mom, 0, 2 * plane * sizeof(double), s));
  FB_CUDA(cudaMemsetAsync(c.d_lec, 0, 4 * plane * sizeof(double), s));
  c.launches += 1 + 2 * (depth - height);
  // upward arrays: moments (forward) or adjoint locals (adjoint)
  double *up1 = adjoint ? c.d_lec + plane : c.d_mom, *up2 = adjoint ? c.d_lec : c.d_mom + plane;
  if (c.d_Q0F && !fp64)
    q2m_kernel<float><<<pt.nLeaves, 256, 0, s>>>(pt.nLeaves, c.n, c.NMleaf, c.NM, c.d_leafStart, c.d_leafCount,
                                                 c.d_leafFmm, c.d_Q0F, c.d_Q1F, sgm, adjoint ? 1 : 0, up1, up2);
  else
    q2m_kernel<double><<<pt.nLeaves, 256, 0, s>>>(pt.nLeaves, c.n, c.NMleaf, c.NM, c.d_leafStart, c.d_leafCount,
                                                  c.d_leafFmm, c.d_Q0, c.d_Q1, sgm, adjoint ? 1 : 0, up1, up2);
  if (marks) cudaEventRecord(marks[0], s);
  for (int lev = depth - 1; lev >= height; lev--) {
    int ordOut = pt.ordMom[lev], ordIn = pt.ordMom[lev + 1];
    const int nOut = nmom(ordOut), nLst = c.h_mOff[nOut];
    const size_t shm = (size_t)kShiftWarps * 5 * nOut * sizeof(double) + (size_t)(nOut + 1 + nLst) * sizeof(int);
    if (shm > 48 * 1024) cudaFuncSetAttribute(m2m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    m2m_kernel<<<pt.fmmLevelCount[lev], kShiftWarps * 32, shm, s>>>(
        pt.fmmLevelStart[lev], pt.fmmLevelCount[lev], c.NM, ordOut, ordIn, c.d_kidFirst, c.d_kidCount, c.d_cubeCtr,
        c.d_mOff, c.d_mLst, nLst, up1, up2);
  }
  if (marks) cudaEventRecord(marks[1], s);
  if (!launch_m2l_only(c, adjoint, fp64)) return false;
  if (marks) cudaEventRecord(marks[2], s);
  // downward arrays: 4 local planes (forward) or the 2 adjoint moment planes
  // plus 2 scratch planes (adjoint)
  double *d1 = adjoint ? c.d_mom : c.d_lec, *d2 = adjoint ? c.d_mom + plane : c.d_lec + plane;
  for (int lev = height; lev < depth; lev++) {
    int ordIn = pt.ordMom[lev], ordOut = pt.ordMom[lev + 1];
    const int nOut = nmom(ordOut), nLst = c.h_lstOff[nOut];
    const size_t shm = (size_t)kShiftWarps * 5 * nmom(ordIn) * sizeof(double) + (size_t)(nOut + 1 + nLst) * sizeof(int);
    if (shm > 48 * 1024) cudaFuncSetAttribute(l2l_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    l2l_kernel<<<ceil_div(pt.fmmLevelCount[lev + 1], kShiftWarps), kShiftWarps * 32, shm, s>>>(
        pt.fmmLevelStart[lev + 1], pt.fmmLevelCount[lev + 1], c.NM, ordIn, ordOut, c.d_fmmParent, c.d_cubeCtr,
        c.d_lstOff, c.d_lst, nLst, d1, d2, c.d_lec + 2 * plane, c.d_lec + 3 * plane);
  }
  if (adjoint) FB_CUDA(cudaMemsetAsync(c.d_lec + 2 * plane, 0, 2 * plane * sizeof(double), s));
  if (marks) cudaEventRecord(marks[3], s);
  FB_CUDA(cudaGetLastError());
  return true;
}

bool launch_m2l_only(Context &c, bool adjoint, bool fp64) {
  if ((adjoint ? c.h_m2lDstT : c.h_m2lDst).empty()) return true;
  FB_DISPATCH_ORDER(c.P, launch_m2l_t, c, adjoint, c.mixed && !fp64);
  c.launches += 1;
  FB_CUDA(cudaGetLastError());
  return true;
}

bool launch_l2p(Context &c, double alpha, double beta, double *out, const double *diagX, double s1, double s2,
                bool adjoint, const double *addend, bool fp64) {
  const size_t plane = (size_t)c.pt.nFmm * c.NM;
  c.launches += 1;
  // adjoint: Q0 . (adjoint dpdn moments + 0) -> dpdn half, Q1 . (adjoint pot moments + 0) -> pot half
  const double *l1 = adjoint ? c.d_mom + plane : c.d_lec, *l2 = c.d_lec + (adjoint ? 2 : 1) * plane;
  const double *l3 = adjoint ? c.d_mom : c.d_lec + 2 * plane, *l4 = c.d_lec + 3 * plane;
  if (c.d_Q0F && !fp64)
    l2p_kernel<float><<<ceil_div(c.n, 256), 256, 0, c.stream>>>(c.n, c.NMleaf, c.NM, c.d_leafOfPanel, c.d_leafFmm,
                                                                c.d_Q0F, c.d_Q1F, l1, l2, l3, l4, alpha, beta,
                                                                c.d_area, diagX, s1, s2, adjoint ? 1 : 0, addend, out);
  else
    l2p_kernel<double><<<ceil_div(c.n, 256), 256, 0, c.stream>>>(c.n, c.NMleaf, c.NM, c.d_leafOfPanel, c.d_leafFmm,
                                                                 c.d_Q0, c.d_Q1, l1, l2, l3, l4, alpha, beta,
                                                                 c.d_area, diagX, s1, s2, adjoint ? 1 : 0, addend,
                                                                 out);
  FB_CUDA(cudaGetLastError());
  return true;
}

}  // namespace fb
