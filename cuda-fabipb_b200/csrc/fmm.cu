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
template <int PM>
__device__ void derivs_inplace(int order, const double *x, double kappa, bool coulombOnly, double *d0, double *dk,
                               int stride) {
  double G0[PM + 2], Gk[PM + 2];
  const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  if (coulombOnly) {
    const double r2 = -1.0 / (r * r);
    G0[0] = kFourPiI / r;
    for (int k = 0; k < order; k++) G0[k + 1] = (2 * k + 1) * r2 * G0[k];
  } else {
    const double rexp = exp(-kappa * r), r1 = 1.0 / r, rr2 = r1 * r1, nr2 = -rr2, k2 = kappa * kappa;
    G0[0] = r1 * kFourPiI;
    Gk[0] = rexp * G0[0];
    G0[1] = nr2 * G0[0];
    Gk[1] = -Gk[0] * (rr2 + kappa * r1);
    for (int k = 1; k < order; k++) {
      G0[k + 1] = (2 * k + 1) * nr2 * G0[k];
      Gk[k + 1] = rr2 * (k2 * Gk[k - 1] - (2 * k + 1) * Gk[k]);
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
      double xa, fb = 0.0;
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
      double v0 = d0[a * stride] * xa;
      if (b >= 0) v0 += d0[b * stride] * fb;
      d0[e * stride] = v0;
      if (!coulombOnly) {
        double vk = dk[a * stride] * xa;
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
__global__ void q2m_kernel(int nLeaves, int n, int NMleaf, int NM, const int *__restrict__ leafStart,
                           const int *__restrict__ leafCount, const int *__restrict__ leafFmm,
                           const double *__restrict__ Q0, const double *__restrict__ Q1,
                           const double *__restrict__ sgm, double *momPot, double *momDpdn) {
  int L = blockIdx.x;
  if (L >= nLeaves) return;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int st = leafStart[L], cnt = leafCount[L], f = leafFmm[L];
  for (int m = warp; m < NMleaf; m += nw) {
    double sp = 0.0, sd = 0.0;
    for (int j = lane; j < cnt; j += 32) {
      sp += Q1[(size_t)m * n + st + j] * sgm[st + j];
      sd += Q0[(size_t)m * n + st + j] * sgm[n + st + j];
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

// M2M: one block per parent cube at one level; threads over output indices
__global__ void m2m_kernel(int first, int count, int NM, int ordOut, int ordIn, const int *__restrict__ kidFirst,
                           const int *__restrict__ kidCount, const double *__restrict__ ctr,
                           const int *__restrict__ lstOff, const int *__restrict__ lst, double *momPot,
                           double *momDpdn) {
  extern __shared__ double sm[];
  double *a = sm, *b1 = sm + NM, *b2 = sm + 2 * NM;
  int f = first + blockIdx.x;
  if (blockIdx.x >= count) return;
  int nOut = nmom(ordOut), nIn = nmom(ordIn);
  double o1 = 0.0, o2 = 0.0;
  int al = threadIdx.x;
  for (int k = 0; k < kidCount[f]; k++) {
    int kid = kidFirst[f] + k;
    double t[3] = {ctr[3 * kid] - ctr[3 * f], ctr[3 * kid + 1] - ctr[3 * f + 1], ctr[3 * kid + 2] - ctr[3 * f + 2]};
    for (int e = threadIdx.x; e < nOut; e += blockDim.x) {
      a[e] = conv_entry(t, e);
      b1[e] = (e < nIn) ? momPot[(size_t)kid * NM + e] : 0.0;
      b2[e] = (e < nIn) ? momDpdn[(size_t)kid * NM + e] : 0.0;
    }
    __syncthreads();
    if (al < nOut) {
      for (int q = lstOff[al]; q < lstOff[al + 1]; q++) {
        int ent = lst[q];
        int ia = ent & 1023, ib = (ent >> 10) & 1023;
        o1 += a[ia] * b1[ib];
        o2 += a[ia] * b2[ib];
      }
    }
    __syncthreads();
  }
  if (al < nOut) {
    momPot[(size_t)f * NM + al] = o1;
    momDpdn[(size_t)f * NM + al] = o2;
  }
}



// M2L: one block (128 threads) per destination cube with a non-empty
// interaction list, sources in batches of 64.  Threads 0..63 each build the
// derivative tensors D^a G0, D^a Gk of one source into shared-memory columns
// while threads 64..127 stage the sign-weighted source moments; then thread
// (alpha, half) accumulates the four local coefficients over half of the batch
// (convM2L: l[alpha] += sum_beta c[beta] veck[alpha+beta]), and the two halves
// are added at the end.  No atomics: every destination cube is one block.
template <int PM>
struct M2LShape {
  static constexpr int NMP = nmom_c(PM);
  static constexpr int B = PM <= 5 ? 64 : 32;               // sources per batch
  static constexpr int S = B + 1;                           // padded column stride
  static constexpr int AP = ((NMP + 31) / 32) * 32;         // threads per half
  static constexpr int T = 2 * (AP > B ? AP : B);           // block size
};

template <int PM>
__global__ void __launch_bounds__(M2LShape<PM>::T)
m2l_kernel(int nDst, const int *__restrict__ dstList, const int *__restrict__ m2lOff,
           const int *__restrict__ m2lSrc, const double *__restrict__ ctr, const int *__restrict__ ordOfCube,
           const int *__restrict__ lstOff, const int *__restrict__ lst, int NM, double kappa, double eps,
           const double *__restrict__ momPot, const double *__restrict__ momDpdn, double *lec1, double *lec2,
           double *lec3, double *lec4) {
  typedef M2LShape<PM> Sh;
  constexpr int NMP = Sh::NMP, B = Sh::B, S = Sh::S, H = Sh::T / 2;
  extern __shared__ double sm[];
  double *sD0 = sm, *sDk = sD0 + NMP * S, *sC1 = sDk + NMP * S, *sC2 = sC1 + NMP * S;
  int *sOff = (int *)(sC2 + NMP * S);
  int *sLst = sOff + NMP + 1;
  if ((int)blockIdx.x >= nDst) return;
  const int f = dstList[blockIdx.x];
  const int order = ordOfCube[f];
  const int nm = ((order + 1) * (order + 2) * (order + 3)) / 6;
  const int o0 = m2lOff[f], o1 = m2lOff[f + 1];
  const int nl = lstOff[NMP];
  for (int i = threadIdx.x; i <= NMP; i += blockDim.x) sOff[i] = lstOff[i];
  for (int i = threadIdx.x; i < nl; i += blockDim.x) sLst[i] = lst[i];
  const int t = threadIdx.x;
  const int al = t % H, half = t / H;
  const int degA = (al < nm) ? c_mi[al].w : 0;
  const double ieps = 1.0 / eps;
  const double cx = ctr[3 * f], cy = ctr[3 * f + 1], cz = ctr[3 * f + 2];
  double l1 = 0.0, l2 = 0.0, l3 = 0.0, l4 = 0.0;
  for (int b0 = o0; b0 < o1; b0 += B) {
    const int nb = min(B, o1 - b0);
    if (t < B) {
      if (t < nb) {
        const int s = m2lSrc[b0 + t];
        const double r[3] = {cx - ctr[3 * s], cy - ctr[3 * s + 1], cz - ctr[3 * s + 2]};
        derivs_inplace<PM>(order, r, kappa, false, sD0 + t, sDk + t, S);
      }
    } else if (t < 2 * B) {
      const int j = t - B;
      if (j < nb) {
        const int s = m2lSrc[b0 + j];
        for (int e = 0; e < nm; e++) {
          const double sg = c_sgn3[e];
          sC1[e * S + j] = sg * momPot[(size_t)s * NM + e];
          sC2[e * S + j] = sg * momDpdn[(size_t)s * NM + e];
        }
      }
    }
    __syncthreads();
    if (al < nm) {
      const int q0 = sOff[al], q1 = sOff[al + 1];
      const int hb = (B + 1) / 2;
      const int j0 = half * hb, j1 = min(nb, j0 + hb);
      for (int q = q0; q < q1; q++) {
        const int ent = sLst[q];
        const int ib = ent & 1023, ig = (ent >> 10) & 1023, db = ent >> 20;
        if (db > order - degA) break;
        const double *pc1 = sC1 + ib * S, *pc2 = sC2 + ib * S;
        const double *p0 = sD0 + ig * S, *pk = sDk + ig * S;
        for (int j = j0; j < j1; j++) {
          const double d0 = p0[j], dk = pk[j], c1 = pc1[j], c2 = pc2[j];
          const double v1 = d0 - dk;
          l1 += c2 * v1;
          l2 += c1 * (eps * dk - d0);
          l3 += c2 * (d0 - dk * ieps);
          l4 -= c1 * v1;
        }
      }
    }
    __syncthreads();
  }
  // combine the two halves (the moment columns are free scratch now)
  if (half == 1 && al < nm) {
    sC1[al] = l1; sC1[H + al] = l2; sC1[2 * H + al] = l3; sC1[3 * H + al] = l4;
  }
  __syncthreads();
  if (half == 0 && al < nm) {
    lec1[(size_t)f * NM + al] += l1 + sC1[al];
    lec2[(size_t)f * NM + al] += l2 + sC1[H + al];
    lec3[(size_t)f * NM + al] += l3 + sC1[2 * H + al];
    lec4[(size_t)f * NM + al] += l4 + sC1[3 * H + al];
  }
}

template <int PM>
size_t m2l_smem_bytes(int nList) {
  typedef M2LShape<PM> Sh;
  return 4 * (size_t)Sh::NMP * Sh::S * sizeof(double) + (Sh::NMP + 1 + nList) * sizeof(int);
}

// L2L: one block per child cube of one level (parents one level up)
__global__ void l2l_kernel(int first, int count, int NM, int ordIn, int ordOut, const int *__restrict__ parent,
                           const double *__restrict__ ctr, const int *__restrict__ lstOff,
                           const int *__restrict__ lst, double *lec1, double *lec2, double *lec3, double *lec4) {
  extern __shared__ double sm[];
  const int nIn = nmom(ordIn), nOut = nmom(ordOut);
  double *a = sm, *i1 = sm + nIn, *i2 = i1 + nIn, *i3 = i2 + nIn, *i4 = i3 + nIn;
  if ((int)blockIdx.x >= count) return;
  const int f = first + blockIdx.x;
  const int p = parent[f];
  const double t[3] = {ctr[3 * f] - ctr[3 * p], ctr[3 * f + 1] - ctr[3 * p + 1], ctr[3 * f + 2] - ctr[3 * p + 2]};
  for (int e = threadIdx.x; e < nIn; e += blockDim.x) {
    a[e] = conv_entry(t, e);
    i1[e] = lec1[(size_t)p * NM + e];
    i2[e] = lec2[(size_t)p * NM + e];
    i3[e] = lec3[(size_t)p * NM + e];
    i4[e] = lec4[(size_t)p * NM + e];
  }
  __syncthreads();
  const int al = threadIdx.x;
  if (al < nOut) {
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
__global__ void l2p_kernel(int n, int NMleaf, int NM, const int *__restrict__ leafOfPanel,
                           const int *__restrict__ leafFmm, const double *__restrict__ Q0,
                           const double *__restrict__ Q1, const double *__restrict__ lec1,
                           const double *__restrict__ lec2, const double *__restrict__ lec3,
                           const double *__restrict__ lec4, double alpha, double beta, const double *__restrict__ area,
                           const double *__restrict__ diagX, double s1, double s2, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t f = (size_t)leafFmm[leafOfPanel[i]] * NM;
  double a = 0.0, b = 0.0;
  for (int m = 0; m < NMleaf; m++) {
    a += Q0[(size_t)m * n + i] * (lec1[f + m] + lec2[f + m]);
    b += Q1[(size_t)m * n + i] * (lec3[f + m] + lec4[f + m]);
  }
  double o0 = (beta == 0.0) ? 0.0 : beta * out[i];
  double o1 = (beta == 0.0) ? 0.0 : beta * out[n + i];
  o0 += alpha * a;
  o1 += alpha * b;
  if (diagX) {
    o0 += s1 * area[i] * diagX[i];
    o1 += s2 * area[i] * diagX[n + i];
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

template <int PM>
static void launch_m2l_t(Context &c) {
  const size_t plane = (size_t)c.pt.nFmm * c.NM;
  const size_t shm = m2l_smem_bytes<PM>(c.nConvList);
  static int attrDone[kMaxOrder + 1] = {0};
  if (!attrDone[PM]) {
    cudaFuncSetAttribute(m2l_kernel<PM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm + 4096);
    attrDone[PM] = 1;
  }
  m2l_kernel<PM><<<(unsigned)c.h_m2lDst.size(), M2LShape<PM>::T, shm, c.stream>>>(
      (int)c.h_m2lDst.size(), c.d_m2lDst, c.d_m2lOff, c.d_m2lSrc, c.d_cubeCtr, c.d_ordM2L, c.d_lstOff, c.d_lst,
      c.NM, c.prm.kappa, c.epsilon, c.d_mom, c.d_mom + plane, c.d_lec, c.d_lec + plane, c.d_lec + 2 * plane,
      c.d_lec + 3 * plane);
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
  // leaf matrices
  if (!c.arena.alloc_n(&c.d_Q0, (size_t)c.NMleaf * c.n) || !c.arena.alloc_n(&c.d_Q1, (size_t)c.NMleaf * c.n))
    return false;
  FB_CHECK(c.leafOrder >= 1, "leaf moment order %d must be >= 1", c.leafOrder);
  FB_DISPATCH_ORDER(c.leafOrder, launch_leaf_moments, c, c.leafOrder);
  FB_CUDA(cudaGetLastError());
  return true;
}

bool launch_far_upward(Context &c, const double *sgm) {
  const PanelTree &pt = c.pt;
  const int depth = pt.t.depth, height = pt.t.height;
  cudaStream_t s = c.stream;
  const size_t plane = (size_t)pt.nFmm * c.NM;
  FB_CUDA(cudaMemsetAsync(c.d_mom, 0, 2 * plane * sizeof(double), s));
  FB_CUDA(cudaMemsetAsync(c.d_lec, 0, 4 * plane * sizeof(double), s));
  c.launches += 1 + 2 * (depth - height);
  q2m_kernel<<<pt.nLeaves, 256, 0, s>>>(pt.nLeaves, c.n, c.NMleaf, c.NM, c.d_leafStart, c.d_leafCount, c.d_leafFmm,
                                        c.d_Q0, c.d_Q1, sgm, c.d_mom, c.d_mom + plane);
  for (int lev = depth - 1; lev >= height; lev--) {
    int ordOut = pt.ordMom[lev], ordIn = pt.ordMom[lev + 1];
    int thr = std::max(32, ((nmom(ordOut) + 31) / 32) * 32);
    size_t shm = 3 * (size_t)nmom(ordOut) * sizeof(double);
    m2m_kernel<<<pt.fmmLevelCount[lev], thr, shm, s>>>(pt.fmmLevelStart[lev], pt.fmmLevelCount[lev], c.NM, ordOut,
                                                       ordIn, c.d_kidFirst, c.d_kidCount, c.d_cubeCtr, c.d_mOff,
                                                       c.d_mLst, c.d_mom, c.d_mom + plane);
  }
  if (!launch_m2l_only(c)) return false;
  for (int lev = height; lev < depth; lev++) {
    int ordIn = pt.ordMom[lev], ordOut = pt.ordMom[lev + 1];
    int thr = std::max(32, ((nmom(ordOut) + 31) / 32) * 32);
    size_t shm = 5 * (size_t)nmom(ordIn) * sizeof(double);
    l2l_kernel<<<pt.fmmLevelCount[lev + 1], thr, shm, s>>>(
        pt.fmmLevelStart[lev + 1], pt.fmmLevelCount[lev + 1], c.NM, ordIn, ordOut, c.d_fmmParent, c.d_cubeCtr,
        c.d_lstOff, c.d_lst, c.d_lec, c.d_lec + plane, c.d_lec + 2 * plane, c.d_lec + 3 * plane);
  }
  FB_CUDA(cudaGetLastError());
  return true;
}

bool launch_m2l_only(Context &c) {
  if (c.h_m2lDst.empty()) return true;
  FB_DISPATCH_ORDER(c.P, launch_m2l_t, c);
  c.launches += 1;
  FB_CUDA(cudaGetLastError());
  return true;
}

bool launch_l2p(Context &c, double alpha, double beta, double *out, const double *diagX, double s1, double s2) {
  const size_t plane = (size_t)c.pt.nFmm * c.NM;
  c.launches += 1;
  l2p_kernel<<<ceil_div(c.n, 256), 256, 0, c.stream>>>(c.n, c.NMleaf, c.NM, c.d_leafOfPanel, c.d_leafFmm, c.d_Q0,
                                                       c.d_Q1, c.d_lec, c.d_lec + plane, c.d_lec + 2 * plane,
                                                       c.d_lec + 3 * plane, alpha, beta, c.d_area, diagX, s1, s2, out);
  FB_CUDA(cudaGetLastError());
  return true;
}

}  // namespace fb
