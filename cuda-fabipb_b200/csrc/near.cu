// near.cu -- Galerkin near field on the device.
//
// The near field couples every panel X of a leaf with every panel Y of each
// leaf in its near list (src/fmm.c:554-593).  With the one-point rule (-q=1,
// the reference default) a disjoint pair is K = Ax*Ay*KER4(mX - mY)
// (src/numQuad.c:586-618 at q=1, src/gpu/gpu_nearfield_cuda.inc:1127-1137);
// pairs that share a vertex, an edge, or are the same panel use the Sauter
// rules instead (src/numQuad.c:401-571).
//
// B200 design:
//   * nothing per pair is stored: each warp owns 32 target panels of one
//     leaf, keeps them in registers, and streams the source panels of every
//     near leaf through a per-warp shared-memory tile, so the P2P work is pure
//     FP32 (or FP64) ALU + two MUFU ops per pair;
//   * positions are stored relative to their own leaf centre, and a target
//     is moved into each source leaf's frame once per leaf pair, which keeps
//     FP32 differences of close panels accurate to ~1e-7 relative;
//   * the coincident pair is masked (r = 0 gives 0), and every pair with a
//     shared vertex carries an FP64 correction "exact Sauter value minus the
//     one-point value" in a CSR table built once on the device, applied in
//     FP64 in the same kernel.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <unordered_map>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "context.cuh"
#include "quad.cuh"

namespace fb {

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
  typedef float4 t;
};
template <>
struct Vec4<double> {
  typedef double4 t;
};
template <typename T>
struct Pair2;
template <>
struct Pair2<float> {
  typedef float2 t;
};
template <>
struct Pair2<double> {
  typedef double2 t;
};

// The ordered kernels' gathers, written so that their loads overlap instead of
// forming one dependent chain per near leaf or special pair.
//
// sym_scratch_sums: the symmetric kernels' sums of this target (offset xo in its
// leaf) over the near-list entries [p0, p1) that they took, in list order:
// the warp reads 32 entries' slots at once and keeps up to 8 scratch loads in
// flight.  take: the lane adds (one lane per target).
template <typename T>
__device__ __forceinline__ void sym_scratch_sums(int p0, int p1, int lane, bool take, int xo,
                                                 const int *__restrict__ symOff, const T *__restrict__ symScr,
                                                 T &a0, T &a1) {
  typedef typename Pair2<T>::t P;
  const P *scr = reinterpret_cast<const P *>(symScr);
  for (int q0 = p0; q0 < p1; q0 += 32) {
    const int o = q0 + lane < p1 ? symOff[q0 + lane] : -1;
    unsigned m = __ballot_sync(0xffffffffu, o >= 0);
    while (m) {   // warp-uniform
      T v0[8], v1[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        v0[u] = v1[u] = (T)0;
        if (m) {   // warp-uniform
          const int oj = __shfl_sync(0xffffffffu, o, __ffs(m) - 1);
          m &= m - 1;
          if (take) {
            const P v = scr[(size_t)oj + xo];
            v0[u] = v.x;
            v1[u] = v.y;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        a0 += v0[u];
        a1 += v1[u];
      }
    }
  }
}

// special_sums: the FP64 special-pair corrections of target X in table order,
// four entries' loads (index, coefficients, then the two densities) at a time.
__device__ __forceinline__ void special_sums(int X, int n, const int *__restrict__ spOff,
                                             const int *__restrict__ spSrc, const double4 *__restrict__ spK,
                                             const double *__restrict__ sgm, double &e0, double &e1) {
  int e = spOff[X];
  const int e1End = spOff[X + 1];
  for (; e + 4 <= e1End; e += 4) {
    int Y[4];
    double4 d[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      Y[u] = spSrc[e + u];
      d[u] = spK[e + u];
    }
    double sp[4], sd[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      sp[u] = sgm[Y[u]];
      sd[u] = sgm[n + Y[u]];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      e0 += d[u].x * sd[u] + d[u].y * sp[u];
      e1 += d[u].z * sd[u] + d[u].w * sp[u];
    }
  }
  for (; e < e1End; e++) {
    const int Y = spSrc[e];
    const double4 d = spK[e];
    const double sp = sgm[Y], sd = sgm[n + Y];
    e0 += d.x * sd + d.y * sp;
    e1 += d.z * sd + d.w * sp;
  }
}

// FP32: the single MUFU instructions (PTX rsqrt.approx / ex2.approx, flush
// to zero; relative error ~2^-22, far below the FP32 P2P tolerance).  FP64:
// the library functions.
__device__ __forceinline__ float rsqrt_t(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
// e^{-kappa r}: float evaluates 2^(kexp r) with kexp = -kappa*log2(e)
__device__ __forceinline__ float expneg_t(float kexp, float r) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(kexp * r));
  return y;
}
__device__ __forceinline__ double expneg_t(double kexp, double r) { return exp(kexp * r); }

template <typename T>
__global__ void near_targets_kernel(int n, const double *__restrict__ vtx, const double *__restrict__ nrm,
                                    const double *__restrict__ area, const int *__restrict__ leafOfPanel,
                                    const double *__restrict__ leafCtr, typename Vec4<T>::t *tgtP,
                                    typename Vec4<T>::t *tgtN) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *v = vtx + 9 * (size_t)i;
  const double *c = leafCtr + 3 * (size_t)leafOfPanel[i];
  double m[3];
  for (int k = 0; k < 3; k++) {
    double a2 = v[3 + k] - v[k], a0 = v[6 + k] - v[3 + k];
    m[k] = v[k] + 0.5 * (a2 + 0.5 * a0);
  }
  typename Vec4<T>::t p, q;
  p.x = (T)(m[0] - c[0]); p.y = (T)(m[1] - c[1]); p.z = (T)(m[2] - c[2]); p.w = (T)area[i];
  q.x = (T)nrm[3 * (size_t)i]; q.y = (T)nrm[3 * (size_t)i + 1]; q.z = (T)nrm[3 * (size_t)i + 2]; q.w = (T)0;
  tgtP[i] = p;
  tgtN[i] = q;
}

// Source records of one apply: {position, A*sigma_dpdn}, {normal, A*sigma_pot}.
// scaleNormal 1 (2): the normal is stored multiplied by the second (first)
// weight, for the packed FP32 kernel, whose pair formula takes the source
// normal only in terms that carry that weight.
template <typename T>
__global__ void near_pack_kernel(int n, const typename Vec4<T>::t *__restrict__ tgtP,
                                 const typename Vec4<T>::t *__restrict__ tgtN, const double *__restrict__ area,
                                 const double *__restrict__ sgm, typename Vec4<T>::t *srcA,
                                 typename Vec4<T>::t *srcB, int scaleNormal) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  typename Vec4<T>::t a = tgtP[i], b = tgtN[i];
  double A = area[i];
  const double wa = A * sgm[n + i], wb = A * sgm[i];
  a.w = (T)wa;  // weight of the dpdn density
  b.w = (T)wb;  // weight of the potential density
  if (scaleNormal) {
    const T w = (T)(scaleNormal == 1 ? wb : wa);
    b.x *= w;
    b.y *= w;
    b.z *= w;
  }
  srcA[i] = a;
  srcB[i] = b;
}

constexpr int kNearWarps = 4;
// resident blocks per SM the register allocation of near_apply_kernel<float> aims at
#ifndef FB_NEAR_MIN_BLOCKS
#define FB_NEAR_MIN_BLOCKS 8
#endif
// FP32 near field with packed f32x2 arithmetic (near_apply_f2_kernel)
#ifndef FB_NEAR_PACKED
#define FB_NEAR_PACKED 1
#endif

// One disjoint pair, one-point rule: the four KER4 kernels (src/kernel.c:109-147)
// at d = target - source, times the source weights a.w = A*sigma_dpdn and
// b.w = A*sigma_pot (the 4 pi and the target area are applied once at the end).
//
// ADJ: the transposed pair block.  With d = target - source, swapping the
// roles of the two panels gives K0 and K3 unchanged, K1(s,t) = -t2 (eps c - 1)
// and K2(s,t) = -t1 (c/eps - 1), so
//   out_pot  += y3 * a.w - t2 (eps c - 1) * b.w
//   out_dpdn += y0 * b.w - t1 (c/eps - 1) * a.w
// with a.w = A*lambda_dpdn and b.w = A*lambda_pot of the source panel.
template <bool ADJ, typename T, typename V>
__device__ __forceinline__ void near_pair(const V a, const V b, T tx, T ty, T tz, const V tn, T kappa, T kexp, T eps,
                                          T ieps, T kap2, T &acc0, T &acc1) {
  const T dx = tx - a.x, dy = ty - a.y, dz = tz - a.z;
  const T r2 = dx * dx + dy * dy + dz * dz;
  const T g = r2 > (T)0 ? rsqrt_t(r2) : (T)0;   // 1/r, 0 for the coincident pair
  const T r = r2 * g;
  const T e = expneg_t(kexp, r);
  const T c = (kappa * r + (T)1) * e;           // (kappa r + 1) e^{-kappa r}
  const T g2 = g * g;
  const T h = g2 * g;
  const T ipX = tn.x * dx + tn.y * dy + tn.z * dz;
  const T ipY = b.x * dx + b.y * dy + b.z * dz;
  const T ip0 = tn.x * b.x + tn.y * b.y + tn.z * b.z;
  const T t1 = ipY * h;                          // dG0/dn_y * 4 pi
  const T t2 = ipX * h;                          // dG0/dn_x * 4 pi
  const T u = ipX * t1;
  const T y0 = g - g * e;                        // G0 - Gk
  const T y1 = t1 * (eps * c - (T)1);            // eps dGk/dn_y - dG0/dn_y
  const T y2 = t2 * (c * ieps - (T)1);           // dGk/dn_x / eps - dG0/dn_x
  const T dd = (ip0 * g - (T)3 * u) * g2;        // d2 G0 / dn_x dn_y
  const T y3 = dd * (c - (T)1) - kap2 * e * u;
  if (ADJ) {
    acc0 += y3 * a.w - t2 * (eps * c - (T)1) * b.w;
    acc1 += y0 * b.w - t1 * (c * ieps - (T)1) * a.w;
  } else {
    acc0 += y0 * a.w + y1 * b.w;
    acc1 += y2 * a.w + y3 * b.w;
  }
}

// One warp per task (leaf L, group of up to 32 target panels).  A full group
// puts one target on each lane; a partial group of mt targets gives each
// target k = 32/mt lanes, which take every k-th source of a tile, and their
// partial sums are added at the end, so short groups keep most lanes busy.
template <typename T, bool ADJ>
__global__ void __launch_bounds__(kNearWarps * 32, sizeof(T) == 4 ? FB_NEAR_MIN_BLOCKS : 1)
near_apply_kernel(int nWork, const int2 *__restrict__ work, const int *__restrict__ leafStart,
                  const int *__restrict__ leafCount, const int *__restrict__ nearOff,
                  const int *__restrict__ nearSrc, const double *__restrict__ leafCtr,
                  const typename Vec4<T>::t *__restrict__ tgtP, const typename Vec4<T>::t *__restrict__ tgtN,
                  const typename Vec4<T>::t *__restrict__ srcA, const typename Vec4<T>::t *__restrict__ srcB,
                  const int *__restrict__ spOff, const int *__restrict__ spSrc,
                  const double4 *__restrict__ spK, const double *__restrict__ sgm,
                  const double *__restrict__ area, int n, T kappa, T kexp, T eps, T ieps, T kap2,
                  double coef, int accumulate, double *out, const int *__restrict__ symOff,
                  const T *__restrict__ symScr) {
  typedef typename Vec4<T>::t V;
  __shared__ V sA[kNearWarps][32];
  __shared__ V sB[kNearWarps][32];
  __shared__ T sR[kNearWarps][2][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int task = blockIdx.x * kNearWarps + warp;
  if (task >= nWork) return;  // warp-uniform
  const int2 wk = work[task];
  const int L = wk.x;
  const int base = leafStart[L], cnt = leafCount[L];
  const int g0 = 32 * wk.y;
  const int mt = min(32, cnt - g0);   // targets in this group
  const int k = 32 / mt;              // lanes per target
  const int t = lane / k, sub = lane - t * k;
  const bool valid = t < mt;
  const int X = base + g0 + (valid ? t : 0);
  const V tp = tgtP[X], tn = tgtN[X];
  const double cx = leafCtr[3 * L], cy = leafCtr[3 * L + 1], cz = leafCtr[3 * L + 2];
  T acc0 = (T)0, acc1 = (T)0;
  const int pBeg = nearOff[L], p1 = nearOff[L + 1];
  // the leaf pairs of the symmetric kernel: their sums for this target are in the scratch
  if (symOff) sym_scratch_sums<T>(pBeg, p1, lane, valid && sub == 0, X - base, symOff, symScr, acc0, acc1);
  // the other near leaves
  for (int p = pBeg; p < p1; p++) {
    if (symOff && symOff[p] >= 0) continue;   // warp-uniform: summed above
    const int S = nearSrc[p];
    const int sb = leafStart[S], sc = leafCount[S];
    const T tx = tp.x + (T)(cx - leafCtr[3 * S]);
    const T ty = tp.y + (T)(cy - leafCtr[3 * S + 1]);
    const T tz = tp.z + (T)(cz - leafCtr[3 * S + 2]);
    for (int j0 = 0; j0 < sc; j0 += 32) {
      const int m = min(32, sc - j0);
      if (lane < m) {
        sA[warp][lane] = srcA[sb + j0 + lane];
        sB[warp][lane] = srcB[sb + j0 + lane];
      }
      __syncwarp();
      if (k == 1) {   // warp-uniform: a full group, unit stride
#pragma unroll 4
        for (int jj = 0; jj < m; jj++)
          near_pair<ADJ>(sA[warp][jj], sB[warp][jj], tx, ty, tz, tn, kappa, kexp, eps, ieps, kap2, acc0, acc1);
      } else {
#pragma unroll 4
        for (int jj = sub; jj < m; jj += k)
          near_pair<ADJ>(sA[warp][jj], sB[warp][jj], tx, ty, tz, tn, kappa, kexp, eps, ieps, kap2, acc0, acc1);
      }
      __syncwarp();
    }
  }
  if (k > 1) {   // warp-uniform: add the k partial sums of each target
    sR[warp][0][lane] = acc0;
    sR[warp][1][lane] = acc1;
    __syncwarp();
    if (valid && sub == 0)
      for (int i = 1; i < k; i++) {
        acc0 += sR[warp][0][lane + i];
        acc1 += sR[warp][1][lane + i];
      }
  }
  if (!valid || sub != 0) return;
  double e0 = 0.0, e1 = 0.0;
  special_sums(X, n, spOff, spSrc, spK, sgm, e0, e1);
  const double AX = area[X] * kFourPiI;
  const double v0 = coef * (AX * (double)acc0 + e0), v1 = coef * (AX * (double)acc1 + e1);
  out[X] = accumulate ? out[X] + v0 : v0;   // each output has exactly one writer
  out[X + n] = accumulate ? out[X + n] + v1 : v1;
}

// ---------------------------------------------------------------------------
// FP32 near field with packed f32x2 arithmetic (sm_100 FFMA2/FMUL2/FADD2):
// every lane evaluates two sources per step, so the issue slots per pair
// drop by about half while the FP32 work stays the same.  A tile of 32
// sources is staged as 16 source pairs, each as four float4
// (-x0 -x1 -y0 -y1 | -z0 -z1 wa0 wa1 | nx0 nx1 ny0 ny1 | nz0 nz1 wb0 wb1),
// so the packed operands come straight from the loads; an odd source count
// is padded with a zero-weight source far away.  Same tasks, lane split,
// pair formula (near_pair) and FP64 epilogue as near_apply_kernel.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// m = w n_s is the source normal multiplied by the weight of the terms it
// enters: wb in the forward block (y1 wb = t1(m) (eps c - 1), y3 wb = dd(m)
// (c - 1) - kap2 e u(m)), wa in the transposed one; so those terms need no
// weight multiply.  SELF (the target's own leaf, the only tile holding the
// coincident pair d = 0): 1/r is taken as 0 there, which zeroes every term.
template <bool ADJ, bool SELF>
__device__ __forceinline__ void near_pair2(const float4 A, const float4 B, const float4 C, const float4 D, float2 tx,
                                           float2 ty, float2 tz, float2 tnx, float2 tny, float2 tnz, float kappa,
                                           float kexp, float eps, float ieps, float kap2, float2 &acc0,
                                           float2 &acc1) {
  const float2 one = f2(1.f), m1 = f2(-1.f);
  const float2 dx = __fadd2_rn(tx, make_float2(A.x, A.y));
  const float2 dy = __fadd2_rn(ty, make_float2(A.z, A.w));
  const float2 dz = __fadd2_rn(tz, make_float2(B.x, B.y));
  const float2 wa = make_float2(B.z, B.w), wb = make_float2(D.z, D.w);
  const float2 mx = make_float2(C.x, C.y), my = make_float2(C.z, C.w), mz = make_float2(D.x, D.y);
  const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
  float2 g;
  if (SELF) {
    g.x = r2.x > 0.f ? rsqrt_t(r2.x) : 0.f;
    g.y = r2.y > 0.f ? rsqrt_t(r2.y) : 0.f;
  } else {   // distinct leaves: distinct panel centroids, r > 0
    g.x = rsqrt_t(r2.x);
    g.y = rsqrt_t(r2.y);
  }
  const float2 r = __fmul2_rn(r2, g);
  const float2 ea = __fmul2_rn(f2(kexp), r);
  float2 e;
  e.x = expneg_t(1.f, ea.x);
  e.y = expneg_t(1.f, ea.y);
  const float2 c = __fmul2_rn(__ffma2_rn(f2(kappa), r, one), e);    // (kappa r + 1) e^{-kappa r}
  const float2 g2 = __fmul2_rn(g, g), h = __fmul2_rn(g2, g);
  const float2 ipX = __ffma2_rn(tnz, dz, __ffma2_rn(tny, dy, __fmul2_rn(tnx, dx)));
  const float2 ipY = __ffma2_rn(mz, dz, __ffma2_rn(my, dy, __fmul2_rn(mx, dx)));     // w n_s.d
  const float2 ip0 = __ffma2_rn(tnz, mz, __ffma2_rn(tny, my, __fmul2_rn(tnx, mx)));  // w n_t.n_s
  const float2 t1 = __fmul2_rn(ipY, h), t2 = __fmul2_rn(ipX, h), u = __fmul2_rn(ipX, t1);
  const float2 y0 = __ffma2_rn(make_float2(-e.x, -e.y), g, g);                       // G0 - Gk
  const float2 dd = __fmul2_rn(__ffma2_rn(u, f2(-3.f), __fmul2_rn(ip0, g)), g2);     // w d2 G0
  const float2 cm1 = __fadd2_rn(c, m1);
  const float2 ke = __fmul2_rn(f2(-kap2), e);
  if (ADJ) {
    // out_pot += y3 wa - t2 (eps c - 1) wb, out_dpdn += y0 wb - t1 (c/eps - 1) wa
    acc0 = __ffma2_rn(dd, cm1, acc0);
    acc0 = __ffma2_rn(ke, u, acc0);
    acc0 = __ffma2_rn(__fmul2_rn(t2, __ffma2_rn(f2(-eps), c, one)), wb, acc0);
    acc1 = __ffma2_rn(y0, wb, acc1);
    acc1 = __ffma2_rn(t1, __ffma2_rn(f2(-ieps), c, one), acc1);
  } else {
    // out_pot += y0 wa + y1 wb, out_dpdn += y2 wa + y3 wb
    acc0 = __ffma2_rn(y0, wa, acc0);
    acc0 = __ffma2_rn(t1, __ffma2_rn(f2(eps), c, m1), acc0);
    acc1 = __ffma2_rn(__fmul2_rn(t2, __ffma2_rn(f2(ieps), c, m1)), wa, acc1);
    acc1 = __ffma2_rn(dd, cm1, acc1);
    acc1 = __ffma2_rn(ke, u, acc1);
  }
}

// one staged tile of up to 32 sources (np packed source pairs) for a target
#ifndef FB_NEAR_UNROLL
#define FB_NEAR_UNROLL 4
#endif
constexpr int kNearUnroll = FB_NEAR_UNROLL;
template <bool ADJ, bool SELF>
__device__ __forceinline__ void near_tile2(const float4 (*sP)[4], int np, int k, int sub, float2 tx, float2 ty,
                                           float2 tz, float2 tnx, float2 tny, float2 tnz, float kappa, float kexp,
                                           float eps, float ieps, float kap2, float2 &acc0, float2 &acc1) {
  if (k == 1) {   // warp-uniform: a full group
#pragma unroll kNearUnroll
    for (int q = 0; q < np; q++)
      near_pair2<ADJ, SELF>(sP[q][0], sP[q][1], sP[q][2], sP[q][3], tx, ty, tz, tnx, tny, tnz, kappa, kexp, eps,
                            ieps, kap2, acc0, acc1);
  } else {
#pragma unroll kNearUnroll
    for (int q = sub; q < np; q += k)
      near_pair2<ADJ, SELF>(sP[q][0], sP[q][1], sP[q][2], sP[q][3], tx, ty, tz, tnx, tny, tnz, kappa, kexp, eps,
                            ieps, kap2, acc0, acc1);
  }
}

template <bool ADJ>
__global__ void __launch_bounds__(kNearWarps * 32, FB_NEAR_MIN_BLOCKS)
near_apply_f2_kernel(int nWork, const int2 *__restrict__ work, const int *__restrict__ leafStart,
                     const int *__restrict__ leafCount, const int *__restrict__ nearOff,
                     const int *__restrict__ nearSrc, const double *__restrict__ leafCtr,
                     const float4 *__restrict__ tgtP, const float4 *__restrict__ tgtN,
                     const float4 *__restrict__ srcA, const float4 *__restrict__ srcB,
                     const int *__restrict__ spOff, const int *__restrict__ spSrc, const double4 *__restrict__ spK,
                     const double *__restrict__ sgm, const double *__restrict__ area, int n, float kappa, float kexp,
                     float eps, float ieps, float kap2, double coef, int accumulate, double *out,
                     const int *__restrict__ symOff, const float2 *__restrict__ symScr) {
  __shared__ float4 sP[kNearWarps][16][4];
  __shared__ float sR[kNearWarps][2][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int task = blockIdx.x * kNearWarps + warp;
  if (task >= nWork) return;  // warp-uniform
  const int2 wk = work[task];
  const int L = wk.x;
  const int base = leafStart[L], cnt = leafCount[L];
  const int g0 = 32 * wk.y;
  const int mt = min(32, cnt - g0);   // targets in this group
  const int k = 32 / mt;              // lanes per target
  const int t = lane / k, sub = lane - t * k;
  const bool valid = t < mt;
  const int X = base + g0 + (valid ? t : 0);
  const float4 tp = tgtP[X], tn = tgtN[X];
  const float2 tnx = f2(tn.x), tny = f2(tn.y), tnz = f2(tn.z);
  const double cx = leafCtr[3 * L], cy = leafCtr[3 * L + 1], cz = leafCtr[3 * L + 2];
  float2 acc0 = f2(0.f), acc1 = f2(0.f);
  float *pf = reinterpret_cast<float *>(&sP[warp][lane >> 1][0]) + (lane & 1);
  const int pBeg = nearOff[L], p1 = nearOff[L + 1];
  // the leaf pairs of the symmetric kernel: their sums for this target are in the scratch
  if (symOff)
    sym_scratch_sums<float>(pBeg, p1, lane, valid && sub == 0, X - base, symOff,
                            reinterpret_cast<const float *>(symScr), acc0.x, acc1.x);
  // the other near leaves
  for (int p = pBeg; p < p1; p++) {
    if (symOff && symOff[p] >= 0) continue;   // warp-uniform: summed above
    const int S = nearSrc[p];
    const int sb = leafStart[S], sc = leafCount[S];
    const float2 tx = f2(tp.x + (float)(cx - leafCtr[3 * S]));
    const float2 ty = f2(tp.y + (float)(cy - leafCtr[3 * S + 1]));
    const float2 tz = f2(tp.z + (float)(cz - leafCtr[3 * S + 2]));
    for (int j0 = 0; j0 < sc; j0 += 32) {
      const int m = min(32, sc - j0);
      float4 a = make_float4(-1e4f, -1e4f, -1e4f, 0.f), b = make_float4(0.f, 0.f, 0.f, 0.f);
      if (lane < m) {
        a = srcA[sb + j0 + lane];
        b = srcB[sb + j0 + lane];
      }
      pf[0] = -a.x; pf[2] = -a.y; pf[4] = -a.z; pf[6] = a.w;
      pf[8] = b.x; pf[10] = b.y; pf[12] = b.z; pf[14] = b.w;
      __syncwarp();
      const int np = (m + 1) >> 1;
      if (S == L)   // warp-uniform
        near_tile2<ADJ, true>(sP[warp], np, k, sub, tx, ty, tz, tnx, tny, tnz, kappa, kexp, eps, ieps, kap2, acc0,
                              acc1);
      else
        near_tile2<ADJ, false>(sP[warp], np, k, sub, tx, ty, tz, tnx, tny, tnz, kappa, kexp, eps, ieps, kap2, acc0,
                               acc1);
      __syncwarp();
    }
  }
  float s0 = acc0.x + acc0.y, s1 = acc1.x + acc1.y;
  if (k > 1) {   // warp-uniform: add the k partial sums of each target
    sR[warp][0][lane] = s0;
    sR[warp][1][lane] = s1;
    __syncwarp();
    if (valid && sub == 0)
      for (int i = 1; i < k; i++) {
        s0 += sR[warp][0][lane + i];
        s1 += sR[warp][1][lane + i];
      }
  }
  if (!valid || sub != 0) return;
  double e0 = 0.0, e1 = 0.0;
  special_sums(X, n, spOff, spSrc, spK, sgm, e0, e1);
  const double AX = area[X] * kFourPiI;
  const double v0 = coef * (AX * (double)s0 + e0), v1 = coef * (AX * (double)s1 + e1);
  out[X] = accumulate ? out[X] + v0 : v0;   // each output has exactly one writer
  out[X + n] = accumulate ? out[X + n] + v1 : v1;
}

// ---------------------------------------------------------------------------
// Symmetric near field (FP32, packed f32x2; mixed contexts; forward and transposed operator).
// The one-point pair term of K(X, Y) and that of K(Y, X) share r, 1/r,
// e^{-kappa r}, (kappa r + 1) e^{-kappa r}, n_X.n_Y and the double-layer
// factors; with d = x_X - x_Y, swapping the panels negates d, so
//   t1(Y,X) = -t2(X,Y),  t2(Y,X) = -t1(X,Y),  u, dd, y0, y3 unchanged,
//   K(Y,X): out_pot  += y0 wa_X - t2 (eps c - 1) wb_X,
//           out_dpdn += -t1 (c/eps - 1) wa_X + y3 wb_X.
// So every unordered pair of distinct near leaves (R, T) is evaluated once
// for both directions.  One warp per leaf pair: the 32-panel groups of R in
// registers (lane = target), T in tiles of 32 staged in shared memory.  In
// step s of a tile, lane t takes the tile's sources (t + s) and (t + s + 16)
// (mod 32), so at every step the 32 lanes hold 32 distinct sources and each
// source's contribution from the lane's target goes to the lane that owns that
// source by two shuffles; after 16 steps every source has had all 32 targets.
// The sums go to a scratch slot per (ordered leaf pair, panel); the ordered
// near-field kernel adds them, in its near-list order, to its own FP32 sums
// (deterministic: no atomics).  Self pairs and pairs with a small leaf stay in
// the ordered kernel.  ADJ: the transposed operator, with the transposed
// blocks of the two directions (near_pair's ADJ terms and their swap).
// ---------------------------------------------------------------------------
#ifndef FB_NEAR_SYM_MIN_BLOCKS
#define FB_NEAR_SYM_MIN_BLOCKS 6
#endif
// leaf pairs whose smaller leaf has fewer panels go to the half-warp kernel (mixed
// contexts, down to FB_NEAR_SYM16_MIN_LEAF panels; larger pairs too where its
// padding saves more than its overhead) or stay in the ordered kernel (FP64)
#ifndef FB_NEAR_SYM_MIN_LEAF
#define FB_NEAR_SYM_MIN_LEAF 48
#endif
#ifndef FB_NEAR_SYM16_MIN_LEAF
#define FB_NEAR_SYM16_MIN_LEAF 4
#endif
#ifndef FB_NEAR_SYM16_COST
#define FB_NEAR_SYM16_COST 125
#endif
#ifndef FB_NEAR_SYM_UNROLL
#define FB_NEAR_SYM_UNROLL 4
#endif
constexpr int kSymUnroll = FB_NEAR_SYM_UNROLL;
constexpr int kSymWarps = 4;

template <bool ADJ>
__device__ __forceinline__ void near_sym_pair2(const float4 A, const float4 B, const float4 C, const float4 D,
                                               float2 tx, float2 ty, float2 tz, float2 tnx, float2 tny, float2 tnz,
                                               float2 wat, float2 wbt, float2 watn, float2 wbtn, float kappa,
                                               float kexp, float eps, float ieps, float kap2, float2 &acc0,
                                               float2 &acc1, float2 &s0, float2 &s1) {
  const float2 one = f2(1.f), m1 = f2(-1.f);
  const float2 dx = __fadd2_rn(tx, make_float2(A.x, A.y));
  const float2 dy = __fadd2_rn(ty, make_float2(A.z, A.w));
  const float2 dz = __fadd2_rn(tz, make_float2(B.x, B.y));
  const float2 wa = make_float2(B.z, B.w), wb = make_float2(D.z, D.w);
  const float2 nx = make_float2(C.x, C.y), ny = make_float2(C.z, C.w), nz = make_float2(D.x, D.y);
  const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
  float2 g;   // distinct leaves: distinct panel centroids, r > 0
  g.x = rsqrt_t(r2.x);
  g.y = rsqrt_t(r2.y);
  const float2 r = __fmul2_rn(r2, g);
  const float2 ea = __fmul2_rn(f2(kexp), r);
  float2 e;
  e.x = expneg_t(1.f, ea.x);
  e.y = expneg_t(1.f, ea.y);
  const float2 c = __fmul2_rn(__ffma2_rn(f2(kappa), r, one), e);    // (kappa r + 1) e^{-kappa r}
  const float2 g2 = __fmul2_rn(g, g), h = __fmul2_rn(g2, g);
  const float2 ipX = __ffma2_rn(tnz, dz, __ffma2_rn(tny, dy, __fmul2_rn(tnx, dx)));   // n_X.d
  const float2 ipY = __ffma2_rn(nz, dz, __ffma2_rn(ny, dy, __fmul2_rn(nx, dx)));      // n_Y.d
  const float2 ip0 = __ffma2_rn(tnz, nz, __ffma2_rn(tny, ny, __fmul2_rn(tnx, nx)));   // n_X.n_Y
  const float2 t1 = __fmul2_rn(ipY, h), t2 = __fmul2_rn(ipX, h), u = __fmul2_rn(ipX, t1);
  const float2 y0 = __ffma2_rn(make_float2(-e.x, -e.y), g, g);                       // G0 - Gk
  const float2 dd = __fmul2_rn(__ffma2_rn(u, f2(-3.f), __fmul2_rn(ip0, g)), g2);     // d2 G0
  const float2 y3 = __ffma2_rn(dd, __fadd2_rn(c, m1), __fmul2_rn(__fmul2_rn(f2(-kap2), e), u));
  const float2 fe = __ffma2_rn(f2(eps), c, m1), fi = __ffma2_rn(f2(ieps), c, m1);    // eps c - 1, c/eps - 1
  const float2 t1fe = __fmul2_rn(t1, fe), t2fi = __fmul2_rn(t2, fi);
  const float2 t2fe = __fmul2_rn(t2, fe), t1fi = __fmul2_rn(t1, fi);
  if (ADJ) {
    // the transposed blocks (near_pair's ADJ terms): K(Y,X)^T to the target X, K(X,Y)^T to the sources
    acc0 = __ffma2_rn(y3, wa, acc0);
    acc0 = __ffma2_rn(make_float2(-t2fe.x, -t2fe.y), wb, acc0);
    acc1 = __ffma2_rn(y0, wb, acc1);
    acc1 = __ffma2_rn(make_float2(-t1fi.x, -t1fi.y), wa, acc1);
    s0 = __ffma2_rn(t1fe, wbt, __fmul2_rn(y3, wat));
    s1 = __ffma2_rn(t2fi, wat, __fmul2_rn(y0, wbt));
  } else {
    // K(X, Y): the target X of this lane, sources Y
    acc0 = __ffma2_rn(y0, wa, acc0);
    acc0 = __ffma2_rn(t1fe, wb, acc0);
    acc1 = __ffma2_rn(t2fi, wa, acc1);
    acc1 = __ffma2_rn(y3, wb, acc1);
    // K(Y, X): the two sources as targets of this lane's panel
    s0 = __ffma2_rn(t2fe, wbtn, __fmul2_rn(y0, wat));
    s1 = __ffma2_rn(t1fi, watn, __fmul2_rn(y3, wbt));
  }
}

template <bool ADJ>
__global__ void __launch_bounds__(kSymWarps * 32, FB_NEAR_SYM_MIN_BLOCKS)
near_sym_f2_kernel(int nTasks, const int4 *__restrict__ tasks, const int *__restrict__ leafStart,
                   const int *__restrict__ leafCount, const double *__restrict__ leafCtr,
                   const float4 *__restrict__ recA, const float4 *__restrict__ recB, float kappa, float kexp,
                   float eps, float ieps, float kap2, float2 *scr) {
  // per warp, component-major: sQ[k][m] holds component k of the tile's sources m and (m + 16) mod 32,
  // interleaved (first, second, first, second), read by lane t at step s from slot (t + s) mod 32
  __shared__ float4 sQ[kSymWarps][4][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int task = blockIdx.x * kSymWarps + warp;
  if (task >= nTasks) return;  // warp-uniform
  const int4 tk = tasks[task];
  const int R = tk.x, T = tk.y;
  const int rb = leafStart[R], rc = leafCount[R], tb = leafStart[T], tc = leafCount[T];
  const float sx = (float)(leafCtr[3 * R] - leafCtr[3 * T]);
  const float sy = (float)(leafCtr[3 * R + 1] - leafCtr[3 * T + 1]);
  const float sz = (float)(leafCtr[3 * R + 2] - leafCtr[3 * T + 2]);
  float4(*Q)[32] = sQ[warp];
  for (int g0 = 0; g0 < rc; g0 += 32) {
    const int t = g0 + lane;
    const bool valid = t < rc;
    // a lane past the group's end: far away, zero weights (its terms vanish, its sums are dropped)
    const float4 a = valid ? recA[rb + t] : make_float4(1e4f, 1e4f, 1e4f, 0.f);
    const float4 b = valid ? recB[rb + t] : make_float4(0.f, 0.f, 1.f, 0.f);
    const float2 tx = f2(a.x + sx), ty = f2(a.y + sy), tz = f2(a.z + sz);
    const float2 tnx = f2(b.x), tny = f2(b.y), tnz = f2(b.z);
    const float2 wat = f2(a.w), wbt = f2(b.w), watn = f2(-a.w), wbtn = f2(-b.w);
    float2 acc0 = f2(0.f), acc1 = f2(0.f);
    for (int j0 = 0; j0 < tc; j0 += 32) {
      const int m = min(32, tc - j0);
      // stage the tile: source j0+lane, or a padding source far away with zero weights
      float4 sa = make_float4(-1e4f, -1e4f, -1e4f, 0.f), sb = make_float4(0.f, 0.f, 1.f, 0.f);
      if (lane < m) {
        sa = recA[tb + j0 + lane];
        sb = recB[tb + j0 + lane];
      }
      // slot m holds source m first and source m + 16 (mod 32, the lane m ^ 16) second
      const float ox = __shfl_xor_sync(0xffffffffu, sa.x, 16), oy = __shfl_xor_sync(0xffffffffu, sa.y, 16);
      const float oz = __shfl_xor_sync(0xffffffffu, sa.z, 16), ow = __shfl_xor_sync(0xffffffffu, sa.w, 16);
      const float px = __shfl_xor_sync(0xffffffffu, sb.x, 16), py = __shfl_xor_sync(0xffffffffu, sb.y, 16);
      const float pz = __shfl_xor_sync(0xffffffffu, sb.z, 16), pw = __shfl_xor_sync(0xffffffffu, sb.w, 16);
      __syncwarp();   // the previous tile's reads are done
      Q[0][lane] = make_float4(-sa.x, -ox, -sa.y, -oy);
      Q[1][lane] = make_float4(-sa.z, -oz, sa.w, ow);
      Q[2][lane] = make_float4(sb.x, px, sb.y, py);
      Q[3][lane] = make_float4(sb.z, pz, sb.w, pw);
      __syncwarp();
      float2 own = f2(0.f);   // this lane's source j0+lane: (pot, dpdn) from the group's 32 targets
#pragma unroll kSymUnroll
      for (int st = 0; st < 16; st++) {
        const int slot = (lane + st) & 31;
        float2 s0, s1;
        near_sym_pair2<ADJ>(Q[0][slot], Q[1][slot], Q[2][slot], Q[3][slot], tx, ty, tz, tnx, tny, tnz, wat, wbt,
                            watn, wbtn, kappa, kexp, eps, ieps, kap2, acc0, acc1, s0, s1);
        // this lane's source was the first source of lane (lane - st) and the second of lane (lane - st - 16)
        const int l1 = (lane - st) & 31, l2 = (lane - st - 16) & 31;
        const float a0 = __shfl_sync(0xffffffffu, s0.x, l1), a1 = __shfl_sync(0xffffffffu, s1.x, l1);
        const float b0 = __shfl_sync(0xffffffffu, s0.y, l2), b1 = __shfl_sync(0xffffffffu, s1.y, l2);
        own = __fadd2_rn(own, __fadd2_rn(make_float2(a0, a1), make_float2(b0, b1)));
      }
      if (lane < m) {   // the tile side's slot: written by the first group, added to by the next
        float2 *q = scr + tk.w + j0 + lane;
        const float2 prev = g0 == 0 ? f2(0.f) : *q;
        *q = __fadd2_rn(prev, own);
      }
    }
    if (valid) scr[tk.z + t] = make_float2(acc0.x + acc0.y, acc1.x + acc1.y);
  }
}

// The symmetric scheme for leaf pairs that pad badly into 32-panel groups
// (mixed contexts; every pair whose smaller leaf has fewer than
// FB_NEAR_SYM_MIN_LEAF panels, and larger ones where 16-panel padding saves
// more than this kernel's per-tile overhead): each half-warp takes its own
// leaf pair with 16-panel groups and 16-source tiles, so a pair of 46-panel
// leaves fills 92% of the lanes instead of the 52% of 32-wide tiles.  In step
// s of a tile, lane t of the half takes sources (t + s) and (t + s + 8)
// (mod 16); after 8 steps every source has had all 16 targets.  Shuffles and
// warp barriers take the half's lane mask, so the two halves may run
// different trip counts.
template <bool ADJ>
__global__ void __launch_bounds__(kSymWarps * 32, FB_NEAR_SYM_MIN_BLOCKS)
near_sym16_f2_kernel(int nTasks, const int4 *__restrict__ tasks, const int *__restrict__ leafStart,
                     const int *__restrict__ leafCount, const double *__restrict__ leafCtr,
                     const float4 *__restrict__ recA, const float4 *__restrict__ recB, float kappa, float kexp,
                     float eps, float ieps, float kap2, float2 *scr) {
  __shared__ float4 sQ[kSymWarps][2][4][16];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
  const unsigned hm = 0xffffu << (16 * half);
  const int task = (blockIdx.x * kSymWarps + warp) * 2 + half;
  if (task >= nTasks) return;  // uniform over the half
  const int4 tk = tasks[task];
  const int R = tk.x, T = tk.y;
  const int rb = leafStart[R], rc = leafCount[R], tb = leafStart[T], tc = leafCount[T];
  const float sx = (float)(leafCtr[3 * R] - leafCtr[3 * T]);
  const float sy = (float)(leafCtr[3 * R + 1] - leafCtr[3 * T + 1]);
  const float sz = (float)(leafCtr[3 * R + 2] - leafCtr[3 * T + 2]);
  float4(*Q)[16] = sQ[warp][half];
  for (int g0 = 0; g0 < rc; g0 += 16) {
    const int t = g0 + hl;
    const bool valid = t < rc;
    // a lane past the group's end: far away, zero weights (its terms vanish, its sums are dropped)
    const float4 a = valid ? recA[rb + t] : make_float4(1e4f, 1e4f, 1e4f, 0.f);
    const float4 b = valid ? recB[rb + t] : make_float4(0.f, 0.f, 1.f, 0.f);
    const float2 tx = f2(a.x + sx), ty = f2(a.y + sy), tz = f2(a.z + sz);
    const float2 tnx = f2(b.x), tny = f2(b.y), tnz = f2(b.z);
    const float2 wat = f2(a.w), wbt = f2(b.w), watn = f2(-a.w), wbtn = f2(-b.w);
    float2 acc0 = f2(0.f), acc1 = f2(0.f);
    // the tile's source j0+hl, or a padding source far away with zero weights; one tile ahead
    float4 na = make_float4(-1e4f, -1e4f, -1e4f, 0.f), nb = make_float4(0.f, 0.f, 1.f, 0.f);
    if (hl < tc) {
      na = recA[tb + hl];
      nb = recB[tb + hl];
    }
    for (int j0 = 0; j0 < tc; j0 += 16) {
      const int m = min(16, tc - j0);
      const float4 sa = na, sb = nb;
      na = make_float4(-1e4f, -1e4f, -1e4f, 0.f);
      nb = make_float4(0.f, 0.f, 1.f, 0.f);
      if (j0 + 16 + hl < tc) {
        na = recA[tb + j0 + 16 + hl];
        nb = recB[tb + j0 + 16 + hl];
      }
      const int js = j0 + (hl < m ? hl : 0);
      const float2 prev = hl < m && g0 > 0 ? scr[tk.w + js] : f2(0.f);
      // slot m holds source m first and source m + 8 (mod 16, the lane m ^ 8) second
      const float ox = __shfl_xor_sync(hm, sa.x, 8), oy = __shfl_xor_sync(hm, sa.y, 8);
      const float oz = __shfl_xor_sync(hm, sa.z, 8), ow = __shfl_xor_sync(hm, sa.w, 8);
      const float px = __shfl_xor_sync(hm, sb.x, 8), py = __shfl_xor_sync(hm, sb.y, 8);
      const float pz = __shfl_xor_sync(hm, sb.z, 8), pw = __shfl_xor_sync(hm, sb.w, 8);
      __syncwarp(hm);   // the previous tile's reads are done
      Q[0][hl] = make_float4(-sa.x, -ox, -sa.y, -oy);
      Q[1][hl] = make_float4(-sa.z, -oz, sa.w, ow);
      Q[2][hl] = make_float4(sb.x, px, sb.y, py);
      Q[3][hl] = make_float4(sb.z, pz, sb.w, pw);
      __syncwarp(hm);
      float2 own = f2(0.f);   // this lane's source j0+hl: (pot, dpdn) from the group's 16 targets
#pragma unroll 4
      for (int st = 0; st < 8; st++) {
        const int slot = (hl + st) & 15;
        float2 s0, s1;
        near_sym_pair2<ADJ>(Q[0][slot], Q[1][slot], Q[2][slot], Q[3][slot], tx, ty, tz, tnx, tny, tnz, wat, wbt,
                            watn, wbtn, kappa, kexp, eps, ieps, kap2, acc0, acc1, s0, s1);
        // this lane's source was the first source of lane (hl - st) and the second of lane (hl - st - 8)
        const int l1 = (hl - st) & 15, l2 = (hl - st - 8) & 15;
        const float a0 = __shfl_sync(hm, s0.x, l1, 16), a1 = __shfl_sync(hm, s1.x, l1, 16);
        const float b0 = __shfl_sync(hm, s0.y, l2, 16), b1 = __shfl_sync(hm, s1.y, l2, 16);
        own = __fadd2_rn(own, __fadd2_rn(make_float2(a0, a1), make_float2(b0, b1)));
      }
      if (hl < m) scr[tk.w + js] = __fadd2_rn(prev, own);   // written by the first group, added to by the next
    }
    if (valid) scr[tk.z + t] = make_float2(acc0.x + acc0.y, acc1.x + acc1.y);
  }
}

// The same symmetric scheme in scalar arithmetic (FP64 contexts): lane t
// takes source (t + s) mod 32 in step s of 32; the source's term from the
// lane's target goes to the owning lane by shuffle.
template <typename T, bool ADJ>
__device__ __forceinline__ void near_sym_pair(const typename Vec4<T>::t a, const typename Vec4<T>::t b, T tx, T ty,
                                              T tz, T tnx, T tny, T tnz, T wat, T wbt, T kappa, T kexp, T eps,
                                              T ieps, T kap2, T &acc0, T &acc1, T &s0, T &s1) {
  const T dx = tx - a.x, dy = ty - a.y, dz = tz - a.z;
  const T r2 = dx * dx + dy * dy + dz * dz;
  const T g = rsqrt_t(r2);   // distinct leaves: r > 0
  const T r = r2 * g;
  const T e = expneg_t(kexp, r);
  const T c = (kappa * r + (T)1) * e;
  const T g2 = g * g, h = g2 * g;
  const T ipX = tnx * dx + tny * dy + tnz * dz;
  const T ipY = b.x * dx + b.y * dy + b.z * dz;
  const T ip0 = tnx * b.x + tny * b.y + tnz * b.z;
  const T t1 = ipY * h, t2 = ipX * h, u = ipX * t1;
  const T y0 = g - g * e;
  const T dd = (ip0 * g - (T)3 * u) * g2;
  const T y3 = dd * (c - (T)1) - kap2 * e * u;
  const T fe = eps * c - (T)1, fi = c * ieps - (T)1;
  if (ADJ) {   // the transposed blocks, as near_pair's ADJ terms
    acc0 += y3 * a.w - t2 * fe * b.w;
    acc1 += y0 * b.w - t1 * fi * a.w;
    s0 = y3 * wat + t1 * fe * wbt;
    s1 = y0 * wbt + t2 * fi * wat;
  } else {
    acc0 += y0 * a.w + t1 * fe * b.w;
    acc1 += t2 * fi * a.w + y3 * b.w;
    s0 = y0 * wat - t2 * fe * wbt;
    s1 = y3 * wbt - t1 * fi * wat;
  }
}

template <typename T, bool ADJ>
__global__ void __launch_bounds__(kSymWarps * 32, sizeof(T) == 8 ? 2 : FB_NEAR_SYM_MIN_BLOCKS)
near_sym_kernel(int nTasks, const int4 *__restrict__ tasks, const int *__restrict__ leafStart,
                const int *__restrict__ leafCount, const double *__restrict__ leafCtr,
                const typename Vec4<T>::t *__restrict__ recA, const typename Vec4<T>::t *__restrict__ recB, T kappa,
                T kexp, T eps, T ieps, T kap2, T *scr) {
  typedef typename Vec4<T>::t V;
  __shared__ V sA[kSymWarps][32], sB[kSymWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int task = blockIdx.x * kSymWarps + warp;
  if (task >= nTasks) return;  // warp-uniform
  const int4 tk = tasks[task];
  const int R = tk.x, Tl = tk.y;
  const int rb = leafStart[R], rc = leafCount[R], tb = leafStart[Tl], tc = leafCount[Tl];
  const T sx = (T)(leafCtr[3 * R] - leafCtr[3 * Tl]);
  const T sy = (T)(leafCtr[3 * R + 1] - leafCtr[3 * Tl + 1]);
  const T sz = (T)(leafCtr[3 * R + 2] - leafCtr[3 * Tl + 2]);
  for (int g0 = 0; g0 < rc; g0 += 32) {
    const int t = g0 + lane;
    const bool valid = t < rc;
    V a, b;
    if (valid) {
      a = recA[rb + t];
      b = recB[rb + t];
    } else {   // far away, zero weights
      a.x = a.y = a.z = (T)1e4; a.w = (T)0;
      b.x = b.y = (T)0; b.z = (T)1; b.w = (T)0;
    }
    const T tx = a.x + sx, ty = a.y + sy, tz = a.z + sz;
    T acc0 = (T)0, acc1 = (T)0;
    for (int j0 = 0; j0 < tc; j0 += 32) {
      const int m = min(32, tc - j0);
      V pa, pb;
      if (lane < m) {
        pa = recA[tb + j0 + lane];
        pb = recB[tb + j0 + lane];
      } else {
        pa.x = pa.y = pa.z = (T)-1e4; pa.w = (T)0;
        pb.x = pb.y = (T)0; pb.z = (T)1; pb.w = (T)0;
      }
      __syncwarp();
      sA[warp][lane] = pa;
      sB[warp][lane] = pb;
      __syncwarp();
      T own0 = (T)0, own1 = (T)0;
#pragma unroll 2
      for (int st = 0; st < 32; st++) {
        const int j = (lane + st) & 31;
        T s0, s1;
        near_sym_pair<T, ADJ>(sA[warp][j], sB[warp][j], tx, ty, tz, b.x, b.y, b.z, a.w, b.w, kappa, kexp, eps, ieps,
                              kap2, acc0, acc1, s0, s1);
        const int from = (lane - st) & 31;   // the lane whose source this step is this lane's
        own0 += __shfl_sync(0xffffffffu, s0, from);
        own1 += __shfl_sync(0xffffffffu, s1, from);
      }
      if (lane < m) {
        T *q = scr + 2 * (size_t)(tk.w + j0 + lane);
        q[0] = (g0 == 0 ? (T)0 : q[0]) + own0;
        q[1] = (g0 == 0 ? (T)0 : q[1]) + own1;
      }
    }
    if (valid) {
      scr[2 * (size_t)(tk.z + t)] = acc0;
      scr[2 * (size_t)(tk.z + t) + 1] = acc1;
    }
  }
}

// FP64 correction for every special pair: exact panelIA0 minus the
// one-point value the P2P loop computes for the same pair.
__global__ void special_coeff_kernel(long long nSp, const int *__restrict__ spDst, const int *__restrict__ spSrc,
                                     const double *__restrict__ vtx, const double *__restrict__ nrm,
                                     const double *__restrict__ area, int q, double kappa, double eps,
                                     double4 *spK, int *caseOut) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nSp) return;
  int Xi = spDst[e], Yi = spSrc[e];
  PanelD X, Y;
  const double *vx = vtx + 9 * (size_t)Xi, *vy = vtx + 9 * (size_t)Yi;
  for (int k = 0; k < 3; k++) {
    for (int c = 0; c < 3; c++) { X.v[k][c] = vx[3 * k + c]; Y.v[k][c] = vy[3 * k + c]; }
  }
  for (int c = 0; c < 3; c++) {
    X.a[0][c] = X.v[2][c] - X.v[1][c]; X.a[1][c] = X.v[0][c] - X.v[2][c]; X.a[2][c] = X.v[1][c] - X.v[0][c];
    Y.a[0][c] = Y.v[2][c] - Y.v[1][c]; Y.a[1][c] = Y.v[0][c] - Y.v[2][c]; Y.a[2][c] = Y.v[1][c] - Y.v[0][c];
    X.n[c] = nrm[3 * (size_t)Xi + c];
    Y.n[c] = nrm[3 * (size_t)Yi + c];
  }
  X.area = area[Xi];
  Y.area = area[Yi];
  double K[4], M[4] = {0, 0, 0, 0};
  int cs = 0;
  panel_ia0_d(q, kappa, eps, X, Y, Xi == Yi, K, &cs);
  if (Xi != Yi) {
    double r[3];
    for (int c = 0; c < 3; c++) {
      double mx = X.v[0][c] + 0.5 * (X.a[2][c] + 0.5 * X.a[0][c]);
      double my = Y.v[0][c] + 0.5 * (Y.a[2][c] + 0.5 * Y.a[0][c]);
      r[c] = mx - my;
    }
    if (r[0] != 0.0 || r[1] != 0.0 || r[2] != 0.0) {
      double y[4];
      ker4_d(kappa, eps, r, X.n, Y.n, y);
      for (int i = 0; i < 4; i++) M[i] = X.area * Y.area * y[i];
    }
  }
  spK[e] = make_double4(K[0] - M[0], K[1] - M[1], K[2] - M[2], K[3] - M[3]);
  if (caseOut) caseOut[e] = cs;
}

// panel i (tree order) as the quadrature rules take it
__device__ inline void load_panel_d(const double *__restrict__ vtx, const double *__restrict__ nrm,
                                    const double *__restrict__ area, int i, PanelD &P) {
  const double *v = vtx + 9 * (size_t)i;
  for (int k = 0; k < 3; k++)
    for (int c = 0; c < 3; c++) P.v[k][c] = v[3 * k + c];
  for (int c = 0; c < 3; c++) {
    P.a[0][c] = P.v[2][c] - P.v[1][c];
    P.a[1][c] = P.v[0][c] - P.v[2][c];
    P.a[2][c] = P.v[1][c] - P.v[0][c];
    P.n[c] = nrm[3 * (size_t)i + c];
  }
  P.area = area[i];
}

// Near field at panel quadrature order q > 1: the reference's near-field loop
// with panelIA0 at order q for every near pair (src/fmm.c:554-593,
// src/numQuad.c:629-697) -- q^4 kernel evaluations for a disjoint pair
// (pnlNil0), the Sauter rules for touching ones -- in FP64, one thread per
// target panel, the near leaves in list order and their panels in order.
// Forward (target X, K = panelIA0(X, Y)):
//   out_pot[X] += K0 s_dpdn[Y] + K1 s_pot[Y],  out_dpdn[X] += K2 s_dpdn[Y] + K3 s_pot[Y].
// ADJ, the transposed operator (target Y, K = panelIA0(X, Y) of the forward
// pair; the near-leaf relation is symmetric):
//   out_pot[Y] += K1 l_pot[X] + K3 l_dpdn[X],  out_dpdn[Y] += K0 l_pot[X] + K2 l_dpdn[X].
template <bool ADJ>
__global__ void __launch_bounds__(128)
near_quad_kernel(int n, int q, const int *__restrict__ leafOfPanel, const int *__restrict__ leafStart,
                 const int *__restrict__ leafCount, const int *__restrict__ nearOff, const int *__restrict__ nearSrc,
                 const double *__restrict__ vtx, const double *__restrict__ nrm, const double *__restrict__ area,
                 double kappa, double eps, const double *__restrict__ sgm, double coef, int accumulate,
                 double *out) {
  const int T = blockIdx.x * blockDim.x + threadIdx.x;
  if (T >= n) return;
  PanelD P;
  load_panel_d(vtx, nrm, area, T, P);
  const int L = leafOfPanel[T];
  double e0 = 0.0, e1 = 0.0;
  const int p1 = nearOff[L + 1];
  for (int p = nearOff[L]; p < p1; p++) {
    const int S = nearSrc[p];
    const int y1 = leafStart[S] + leafCount[S];
    for (int Y = leafStart[S]; Y < y1; Y++) {
      PanelD Q;
      load_panel_d(vtx, nrm, area, Y, Q);
      double K[4];
      const double sp = sgm[Y], sd = sgm[n + Y];
      if (ADJ) {
        panel_ia0_d(q, kappa, eps, Q, P, Y == T, K, nullptr);
        e0 += K[1] * sp + K[3] * sd;
        e1 += K[0] * sp + K[2] * sd;
      } else {
        panel_ia0_d(q, kappa, eps, P, Q, Y == T, K, nullptr);
        e0 += K[0] * sd + K[1] * sp;
        e1 += K[2] * sd + K[3] * sp;
      }
    }
  }
  const double v0 = coef * e0, v1 = coef * e1;
  out[T] = accumulate ? out[T] + v0 : v0;   // each output has exactly one writer
  out[T + n] = accumulate ? out[T + n] + v1 : v1;
}

namespace {

struct VKey {
  uint64_t a, b, c;
  bool operator==(const VKey &o) const { return a == o.a && b == o.b && c == o.c; }
};
struct VKeyHash {
  size_t operator()(const VKey &k) const {
    uint64_t h = k.a * 0x9E3779B97F4A7C15ULL;
    h ^= k.b + 0x7F4A7C159E3779B9ULL + (h << 6) + (h >> 2);
    h ^= k.c + 0x94D049BB133111EBULL + (h << 6) + (h >> 2);
    return (size_t)h;
  }
};
inline uint64_t dbits(double v) {
  if (v == 0.0) v = 0.0;  // -0.0 and 0.0 compare equal in nrCommonVtx
  uint64_t u;
  memcpy(&u, &v, 8);
  return u;
}

}  // namespace

// ---------------------------------------------------------------------------
// Special-pair search on the device: the panels sharing a vertex with X (by
// exact coordinates, -0.0 = 0.0, as nrCommonVtx, src/numQuad.c:312), X itself,
// kept when their leaves are near, ascending, as CSR by X.  The 3N corners are
// sorted by a 64-bit hash of their coordinates; equal-hash runs are checked
// for exact equality (a collision sends the search to the host path, as does
// a panel with more than kSpCand candidates).
// ---------------------------------------------------------------------------
constexpr int kSpCand = 64;

__device__ __forceinline__ unsigned long long vtx_bits(double v) {
  return (unsigned long long)__double_as_longlong(v == 0.0 ? 0.0 : v);
}
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {   // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__global__ void corner_keys_kernel(int nc, const double *__restrict__ vtx, unsigned long long *keys, int *vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const double *x = vtx + 3 * (size_t)i;   // corner i = vertex i%3 of panel i/3
  keys[i] = mix64(vtx_bits(x[0]) + mix64(vtx_bits(x[1]) + mix64(vtx_bits(x[2]))));
  vals[i] = i;
}

__global__ void corner_runs_kernel(int nc, const unsigned long long *__restrict__ keys, const int *__restrict__ vals,
                                   const double *__restrict__ vtx, int *flag, int *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nc) return;
  int f = 1;
  if (p > 0 && keys[p] == keys[p - 1]) {
    f = 0;
    const double *a = vtx + 3 * (size_t)vals[p], *b = vtx + 3 * (size_t)vals[p - 1];
    for (int k = 0; k < 3; k++)
      if (vtx_bits(a[k]) != vtx_bits(b[k])) atomicExch(err, 1);   // hash collision
  }
  flag[p] = f;
}

// gid: inclusive scan of the run flags (group g = gid - 1)
__global__ void corner_groups_kernel(int nc, const int *__restrict__ flag, const int *__restrict__ gid,
                                     const int *__restrict__ vals, int *gStart, int *cornerGroup) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nc) return;
  const int g = gid[p] - 1;
  if (flag[p]) gStart[g] = p;
  if (p == nc - 1) gStart[g + 1] = nc;
  cornerGroup[vals[p]] = g;
}

// WRITE = false: count per panel into cnt; true: write the sources at off[X]
template <bool WRITE>
__global__ void special_pairs_kernel(int n, const int *__restrict__ cornerGroup, const int *__restrict__ gStart,
                                     const int *__restrict__ vals, const int *__restrict__ leafOf,
                                     const int *__restrict__ nearOff, const int *__restrict__ nearSorted, int *cnt,
                                     const int *__restrict__ off, int *spSrc, int *spDst, int *err) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  if (X >= n) return;
  int cand[kSpCand];
  int m = 0;
  cand[m++] = X;
  for (int k = 0; k < 3; k++) {
    const int g = cornerGroup[3 * X + k];
    for (int p = gStart[g]; p < gStart[g + 1]; p++) {
      if (m == kSpCand) {
        atomicExch(err, 2);
        if (!WRITE) cnt[X] = 0;
        return;
      }
      cand[m++] = vals[p] / 3;
    }
  }
  for (int i = 1; i < m; i++) {   // insertion sort of the few candidates
    const int v = cand[i];
    int j = i - 1;
    while (j >= 0 && cand[j] > v) {
      cand[j + 1] = cand[j];
      j--;
    }
    cand[j + 1] = v;
  }
  const int L = leafOf[X];
  const int *ns = nearSorted + nearOff[L];
  const int nn = nearOff[L + 1] - nearOff[L];
  int o = WRITE ? off[X] : 0, c = 0;
  for (int i = 0; i < m; i++) {
    if (i > 0 && cand[i] == cand[i - 1]) continue;
    const int Y = cand[i], LY = leafOf[Y];
    int lo = 0, hi = nn;   // LY in the sorted near list of L?
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ns[mid] < LY) lo = mid + 1;
      else hi = mid;
    }
    if (lo < nn && ns[lo] == LY) {
      if (WRITE) {
        spSrc[o] = Y;
        spDst[o] = X;
        o++;
      }
      c++;
    }
  }
  if (!WRITE) cnt[X] = c;
}

// 1: tables built (c.d_spOff, c.d_spSrc, *d_spDst, c.nSpecial); 0: use the
// host search instead; -1: CUDA error (message set)
static int special_pairs_device(Context &c, const std::vector<int> &nearSortedFlat, int **d_spDst) {
  const int n = c.n, nc = 3 * n;
  cudaStream_t s = c.stream;
  DevArena tmp;
  unsigned long long *keys = nullptr, *keysS = nullptr;
  int *vals = nullptr, *valsS = nullptr, *flag = nullptr, *gid = nullptr, *cornerGroup = nullptr, *gStart = nullptr;
  int *cnt = nullptr, *err = nullptr, *d_nearSorted = nullptr;
  if (!tmp.alloc_n(&keys, nc) || !tmp.alloc_n(&keysS, nc) || !tmp.alloc_n(&vals, nc) || !tmp.alloc_n(&valsS, nc) ||
      !tmp.alloc_n(&flag, nc) || !tmp.alloc_n(&gid, nc) || !tmp.alloc_n(&cornerGroup, nc) ||
      !tmp.alloc_n(&gStart, (size_t)nc + 1) || !tmp.alloc_n(&cnt, (size_t)n + 1) || !tmp.alloc_n(&err, 1) ||
      !tmp.upload(&d_nearSorted, nearSortedFlat, s))
    return -1;
  FB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  size_t tb1 = 0, tb2 = 0, tb3 = 0;
  FB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb1, keys, keysS, vals, valsS, nc, 0, 64, s));
  FB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb2, flag, gid, nc, s));
  FB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb3, cnt, cnt, n + 1, s));
  void *tbuf = nullptr;
  if (!tmp.alloc(&tbuf, std::max(tb1, std::max(tb2, tb3)))) return -1;
  const size_t tbytes = std::max(tb1, std::max(tb2, tb3));
  corner_keys_kernel<<<ceil_div(nc, 256), 256, 0, s>>>(nc, c.d_vtx, keys, vals);
  size_t tb = tbytes;
  FB_CUDA(cub::DeviceRadixSort::SortPairs(tbuf, tb, keys, keysS, vals, valsS, nc, 0, 64, s));
  corner_runs_kernel<<<ceil_div(nc, 256), 256, 0, s>>>(nc, keysS, valsS, c.d_vtx, flag, err);
  tb = tbytes;
  FB_CUDA(cub::DeviceScan::InclusiveSum(tbuf, tb, flag, gid, nc, s));
  corner_groups_kernel<<<ceil_div(nc, 256), 256, 0, s>>>(nc, flag, gid, valsS, gStart, cornerGroup);
  special_pairs_kernel<false><<<ceil_div(n, 128), 128, 0, s>>>(n, cornerGroup, gStart, valsS, c.d_leafOfPanel,
                                                               c.d_nearOff, d_nearSorted, cnt, nullptr, nullptr,
                                                               nullptr, err);
  FB_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int), s));
  if (!c.arena.alloc_n(&c.d_spOff, (size_t)n + 1)) return -1;
  tb = tbytes;
  FB_CUDA(cub::DeviceScan::ExclusiveSum(tbuf, tb, cnt, c.d_spOff, n + 1, s));
  int hErr = 0, total = 0;
  FB_CUDA(cudaMemcpyAsync(&hErr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaMemcpyAsync(&total, c.d_spOff + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaStreamSynchronize(s));
  FB_CUDA(cudaGetLastError());
  if (hErr) return 0;
  c.nSpecial = total;
  if (!c.arena.alloc_n(&c.d_spSrc, (size_t)std::max(total, 1)) || !c.arena.alloc_n(d_spDst, (size_t)std::max(total, 1)))
    return -1;
  special_pairs_kernel<true><<<ceil_div(n, 128), 128, 0, s>>>(n, cornerGroup, gStart, valsS, c.d_leafOfPanel,
                                                              c.d_nearOff, d_nearSorted, nullptr, c.d_spOff,
                                                              c.d_spSrc, *d_spDst, err);
  FB_CUDA(cudaGetLastError());
  FB_CUDA(cudaStreamSynchronize(s));   // the temporaries are freed on return
  return 1;
}

static bool special_pairs_host(Context &c, const std::vector<int> &nearSortedFlat, int **d_spDst);
static bool setup_near_targets(Context &c);

bool setup_near(Context &c) {
  const PanelTree &pt = c.pt;
  cudaStream_t s = c.stream;
  // -q=1: the one-point P2P kernels plus the FP64 special-pair corrections;
  // -q>1: near_quad_kernel (panelIA0 at order q for every near pair).  The
  // special-pair table is built at order q either way (the preconditioners
  // assemble their blocks from it).
  if (c.prm.quad_order < 1 || c.prm.quad_order > 10) {
    set_error("panel quadrature order -q=%d outside 1..10", c.prm.quad_order);
    return false;
  }
  // the direct operator: every leaf is near every leaf
  if (c.dense) {
    PanelTree &w = c.pt;
    w.nearOff.assign(w.nLeaves + 1, 0);
    w.nearSrc.clear();
    w.nearDst.clear();
    for (int L = 0; L < w.nLeaves; L++) {
      w.nearOff[L] = (int)w.nearSrc.size();
      for (int S = 0; S < w.nLeaves; S++) { w.nearSrc.push_back(S); w.nearDst.push_back(L); }
    }
    w.nearOff[w.nLeaves] = (int)w.nearSrc.size();
    if (!c.arena.upload(&c.d_nearOff, w.nearOff, s) || !c.arena.upload(&c.d_nearSrc, w.nearSrc, s)) return false;
  }
  // warp tasks: (leaf, group of 32 targets), the most expensive first so the
  // last wave of the grid holds the short tasks (a warp's time ~ sources / k,
  // k = lanes per target)
  std::vector<int2> work;
  std::vector<long long> cost;
  c.maxLeaf = 0;
  c.nearPanelPairs = 0;
  for (int L = 0; L < pt.nLeaves; L++) {
    int cnt = pt.leafCount[L];
    c.maxLeaf = std::max(c.maxLeaf, cnt);
    long long srcs = 0;
    for (int p = pt.nearOff[L]; p < pt.nearOff[L + 1]; p++) srcs += pt.leafCount[pt.nearSrc[p]];
    c.nearPanelPairs += srcs * cnt;
    for (int g = 0; g * 32 < cnt; g++) {
      work.push_back(make_int2(L, g));
      cost.push_back(srcs / (32 / std::min(32, cnt - 32 * g)));
    }
  }
  {
    std::vector<int> ord(work.size());
    for (size_t i = 0; i < ord.size(); i++) ord[i] = (int)i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<int2> sorted(work.size());
    for (size_t i = 0; i < ord.size(); i++) sorted[i] = work[ord[i]];
    work.swap(sorted);
  }
  c.nWork = (int)work.size();
  if (!c.arena.upload(&c.d_work, work, s)) return false;

  StageTimer tm("near_setup", s);
  // special pairs: panels sharing a vertex (exact coordinates), restricted to
  // near leaf pairs, plus the panel itself -- on the device, or on the host
  // when the device search declines
  std::vector<int> nearSortedFlat(pt.nearSrc.size());
  for (int L = 0; L < pt.nLeaves; L++) {
    std::copy(pt.nearSrc.begin() + pt.nearOff[L], pt.nearSrc.begin() + pt.nearOff[L + 1],
              nearSortedFlat.begin() + pt.nearOff[L]);
    std::sort(nearSortedFlat.begin() + pt.nearOff[L], nearSortedFlat.begin() + pt.nearOff[L + 1]);
  }
  int *d_spDst = nullptr;
  // FABIPB_B200_HOST_SPECIAL=1 forces the host search (the tests compare the two)
  const int onDevice = getenv("FABIPB_B200_HOST_SPECIAL") ? 0 : special_pairs_device(c, nearSortedFlat, &d_spDst);
  if (onDevice < 0) return false;
  if (onDevice == 0 && !special_pairs_host(c, nearSortedFlat, &d_spDst)) return false;
  tm.mark("special_pairs");
  if (!c.arena.alloc_n(&c.d_spK, (size_t)std::max<long long>(c.nSpecial, 1))) return false;
  if (c.nSpecial > 0) {
    special_coeff_kernel<<<ceil_div(c.nSpecial, 128), 128, 0, s>>>(
        c.nSpecial, d_spDst, c.d_spSrc, c.d_vtx, c.d_nrm, c.d_area, c.prm.quad_order, c.prm.kappa,
        c.epsilon, c.d_spK, nullptr);
    FB_CUDA(cudaGetLastError());
  }
  tm.mark("special_coeff");
  return setup_near_targets(c);
}

// The host search (used when the device search declines): vertex ids from a
// hash map of exact coordinates, per panel its sharing panels, on host threads.
static bool special_pairs_host(Context &c, const std::vector<int> &nearSortedFlat, int **d_spDst) {
  const PanelTree &pt = c.pt;
  const int n = c.n;
  cudaStream_t s = c.stream;
  if (c.h_vtx.size() != 9 * (size_t)n) {   // the device tree keeps the tree-order panels on the device only
    c.h_vtx.resize(9 * (size_t)n);
    FB_CUDA(cudaMemcpyAsync(c.h_vtx.data(), c.d_vtx, 9 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
  }
  std::unordered_map<VKey, int, VKeyHash> vid;
  vid.reserve((size_t)n * 2);
  std::vector<int> pv(3 * (size_t)n);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      const double *x = &c.h_vtx[9 * (size_t)i + 3 * k];
      VKey key{dbits(x[0]), dbits(x[1]), dbits(x[2])};
      auto it = vid.find(key);
      int id;
      if (it == vid.end()) {
        id = (int)vid.size();
        vid.emplace(key, id);
      } else {
        id = it->second;
      }
      pv[3 * (size_t)i + k] = id;
    }
  const int nv = (int)vid.size();
  std::vector<int> vOff(nv + 1, 0), vPan(3 * (size_t)n);
  for (int i = 0; i < 3 * n; i++) vOff[pv[i] + 1]++;
  for (int v = 0; v < nv; v++) vOff[v + 1] += vOff[v];
  {
    std::vector<int> cur(vOff.begin(), vOff.end() - 1);
    for (int i = 0; i < 3 * n; i++) vPan[cur[pv[i]]++] = i / 3;
  }
  std::vector<int> leafOf(n);
  for (int L = 0; L < pt.nLeaves; L++)
    for (int k = 0; k < pt.leafCount[L]; k++) leafOf[pt.leafStart[L] + k] = L;
  // per panel: itself and the panels sharing a vertex with it, ascending,
  // kept when their leaves are near; chunks of panels on host threads, merged
  // in panel order
  std::vector<int> spOff(n + 1, 0), spDst, spSrc;
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::vector<int>> partSrc(nth);
  std::vector<int> cntOf(n, 0);
  auto work_range = [&](int th) {
    const int x0 = (int)((long long)n * th / nth), x1 = (int)((long long)n * (th + 1) / nth);
    std::vector<int> cand;
    std::vector<int> &out = partSrc[th];
    out.reserve(16 * (size_t)(x1 - x0));
    for (int X = x0; X < x1; X++) {
      cand.clear();
      cand.push_back(X);
      for (int k = 0; k < 3; k++) {
        int v = pv[3 * (size_t)X + k];
        for (int e = vOff[v]; e < vOff[v + 1]; e++) cand.push_back(vPan[e]);
      }
      std::sort(cand.begin(), cand.end());
      cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
      const int *nb = nearSortedFlat.data() + pt.nearOff[leafOf[X]];
      const int *ne = nearSortedFlat.data() + pt.nearOff[leafOf[X] + 1];
      int cnt = 0;
      for (int Y : cand)
        if (std::binary_search(nb, ne, leafOf[Y])) {
          out.push_back(Y);
          cnt++;
        }
      cntOf[X] = cnt;
    }
  };
  {
    std::vector<std::thread> pool;
    for (int th = 1; th < nth; th++) pool.emplace_back(work_range, th);
    work_range(0);
    for (auto &th : pool) th.join();
  }
  for (int X = 0; X < n; X++) spOff[X + 1] = spOff[X] + cntOf[X];
  spSrc.reserve(spOff[n]);
  for (int th = 0; th < nth; th++) spSrc.insert(spSrc.end(), partSrc[th].begin(), partSrc[th].end());
  spDst.resize(spSrc.size());
  for (int X = 0; X < n; X++)
    for (int e = spOff[X]; e < spOff[X + 1]; e++) spDst[e] = X;
  c.nSpecial = (long long)spSrc.size();
  if (!c.arena.upload(&c.d_spOff, spOff, s)) return false;
  if (!c.arena.upload(&c.d_spSrc, spSrc, s)) return false;
  if (!c.arena.upload(d_spDst, spDst, s)) return false;
  return true;
}

// The symmetric kernels' leaf pairs (FMM operator, both precisions): every
// unordered pair of distinct near leaves whose smaller leaf has at least
// FB_NEAR_SYM_MIN_LEAF panels, the larger leaf on the register side; a scratch
// slot of 2 floats per (ordered pair, target panel); costliest pairs first.
// FABIPB_B200_NEAR_SYM=0 turns it off (every pair in the ordered kernel).
static bool setup_near_sym(Context &c) {
  c.nSymTasks = 0;
  const char *env = getenv("FABIPB_B200_NEAR_SYM");
  if (c.dense || (env && atoi(env) == 0)) return true;
  const PanelTree &pt = c.pt;
  const size_t nEnt = pt.nearSrc.size();
  std::vector<int> symOff(nEnt, -1);
  std::vector<int4> tasks;
  std::vector<long long> cost;
  std::vector<char> half;   // a pair with a small leaf: near_sym16_f2_kernel
  long long tot = 0, pairs = 0;
  for (int L = 0; L < pt.nLeaves; L++)
    for (int p = pt.nearOff[L]; p < pt.nearOff[L + 1]; p++) {
      const int S = pt.nearSrc[p];
      if (S <= L) continue;
      const int cl = pt.leafCount[L], cs = pt.leafCount[S];
      const int mn = std::min(cl, cs);
      if (mn < (c.mixed ? FB_NEAR_SYM16_MIN_LEAF : FB_NEAR_SYM_MIN_LEAF)) continue;
      // mixed contexts: the half-warp kernel where its padding to 16-panel groups and tiles saves
      // more than its larger per-tile overhead (FB_NEAR_SYM16_COST percent of the 32-wide cost
      // per padded pair), which always holds below FB_NEAR_SYM_MIN_LEAF
      const long long p32 = (long long)((cl + 31) / 32) * ((cs + 31) / 32) * 1024;
      const long long p16 = (long long)((cl + 15) / 16) * ((cs + 15) / 16) * 256;
      const bool small = c.mixed && (mn < FB_NEAR_SYM_MIN_LEAF || p16 * FB_NEAR_SYM16_COST < p32 * 100);
      int q = -1;   // the mirror entry (S <- L)
      for (int k = pt.nearOff[S]; k < pt.nearOff[S + 1]; k++)
        if (pt.nearSrc[k] == L) { q = k; break; }
      if (q < 0) continue;   // not mirrored: both directions stay ordered
      const bool lReg = cl >= cs;
      const int R = lReg ? L : S, T = lReg ? S : L, pR = lReg ? p : q, pT = lReg ? q : p;
      FB_CHECK(tot + cl + cs < 2147483647LL, "symmetric near-field scratch above 2^31 slots");
      symOff[pR] = (int)tot;
      tot += pt.leafCount[R];
      symOff[pT] = (int)tot;
      tot += pt.leafCount[T];
      tasks.push_back(make_int4(R, T, symOff[pR], symOff[pT]));
      cost.push_back((long long)cl * cs);
      half.push_back(small);
      pairs += (long long)cl * cs;
    }
  if (tasks.empty()) return true;
  // the 32-wide tasks first, then the half-warp ones, each by decreasing cost
  std::vector<int> ord(tasks.size());
  for (size_t i = 0; i < ord.size(); i++) ord[i] = (int)i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    return half[a] != half[b] ? half[b] != 0 : cost[a] > cost[b];
  });
  std::vector<int4> sorted(tasks.size());
  int n32 = 0;
  for (size_t i = 0; i < ord.size(); i++) {
    sorted[i] = tasks[ord[i]];
    n32 += half[ord[i]] ? 0 : 1;
  }
  cudaStream_t s = c.stream;
  const size_t esz = c.mixed ? sizeof(float) : sizeof(double);   // scratch element; records are 4 of them
  if (!c.arena.upload(&c.d_symTask, sorted, s) || !c.arena.upload(&c.d_symOff, symOff, s) ||
      !c.arena.alloc(&c.d_symScr, 2 * esz * (size_t)tot) || !c.arena.alloc(&c.d_symA, 4 * esz * (size_t)c.n) ||
      !c.arena.alloc(&c.d_symB, 4 * esz * (size_t)c.n))
    return false;
  c.nSymTasks = (int)sorted.size();
  c.nSym32 = n32;
  c.symPanelPairs = pairs;
  return true;
}

// static target geometry relative to the leaf centres
static bool setup_near_targets(Context &c) {
  const int n = c.n;
  cudaStream_t s = c.stream;
  size_t vb = c.mixed ? sizeof(float4) : sizeof(double4);
  if (!c.arena.alloc(&c.d_tgtP, vb * n) || !c.arena.alloc(&c.d_tgtN, vb * n) ||
      !c.arena.alloc(&c.d_srcA, vb * n) || !c.arena.alloc(&c.d_srcB, vb * n))
    return false;
  if (c.mixed) {
    near_targets_kernel<float><<<ceil_div(n, 256), 256, 0, s>>>(
        n, c.d_vtx, c.d_nrm, c.d_area, c.d_leafOfPanel, c.d_leafCtr, (float4 *)c.d_tgtP, (float4 *)c.d_tgtN);
  } else {
    near_targets_kernel<double><<<ceil_div(n, 256), 256, 0, s>>>(
        n, c.d_vtx, c.d_nrm, c.d_area, c.d_leafOfPanel, c.d_leafCtr, (double4 *)c.d_tgtP, (double4 *)c.d_tgtN);
  }
  FB_CUDA(cudaGetLastError());
  return setup_near_sym(c);
}

template <typename T, bool ADJ>
static void launch_near_t(Context &c, const void *tgtP, const void *tgtN, void *srcA, void *srcB, const double *sgm,
                          double coef, double *out, cudaStream_t s, bool accumulate) {
  typedef typename Vec4<T>::t V;
  const int n = c.n;
  const double kap = c.prm.kappa, eps = c.epsilon;
  const unsigned grid = ceil_div(c.nWork, kNearWarps);
  const double kexp = sizeof(T) == 4 ? -kap * 1.4426950408889634 : -kap;   // float: exp2 argument
  const bool packed = sizeof(T) == 4 && FB_NEAR_PACKED;
  near_pack_kernel<T><<<ceil_div(n, 256), 256, 0, s>>>(n, (const V *)tgtP, (const V *)tgtN, c.d_area, sgm, (V *)srcA,
                                                       (V *)srcB, packed ? (ADJ ? 2 : 1) : 0);
  if (packed) {
    const bool sym = c.nSymTasks > 0 && tgtP == c.d_tgtP;
    if (sym) {   // unordered leaf pairs of the symmetric kernel first, into the scratch
      near_pack_kernel<float><<<ceil_div(n, 256), 256, 0, s>>>(n, (const float4 *)tgtP, (const float4 *)tgtN,
                                                               c.d_area, sgm, (float4 *)c.d_symA, (float4 *)c.d_symB, 0);
      if (c.nSym32 > 0) {
        near_sym_f2_kernel<ADJ><<<ceil_div(c.nSym32, kSymWarps), kSymWarps * 32, 0, s>>>(
            c.nSym32, c.d_symTask, c.d_leafStart, c.d_leafCount, c.d_leafCtr, (const float4 *)c.d_symA,
            (const float4 *)c.d_symB, (float)kap, (float)kexp, (float)eps, (float)(1.0 / eps), (float)(kap * kap),
            (float2 *)c.d_symScr);
        c.launches += 1;
      }
      if (c.nSymTasks > c.nSym32) {
        near_sym16_f2_kernel<ADJ><<<ceil_div(c.nSymTasks - c.nSym32, 2 * kSymWarps), kSymWarps * 32, 0, s>>>(
            c.nSymTasks - c.nSym32, c.d_symTask + c.nSym32, c.d_leafStart, c.d_leafCount, c.d_leafCtr,
            (const float4 *)c.d_symA, (const float4 *)c.d_symB, (float)kap, (float)kexp, (float)eps,
            (float)(1.0 / eps), (float)(kap * kap), (float2 *)c.d_symScr);
        c.launches += 1;
      }
      c.launches += 1;
    }
    near_apply_f2_kernel<ADJ><<<grid, kNearWarps * 32, 0, s>>>(
        c.nWork, c.d_work, c.d_leafStart, c.d_leafCount, c.d_nearOff, c.d_nearSrc, c.d_leafCtr,
        (const float4 *)tgtP, (const float4 *)tgtN, (const float4 *)srcA, (const float4 *)srcB, c.d_spOff, c.d_spSrc,
        ADJ ? c.d_spKT : c.d_spK, sgm, c.d_area, n, (float)kap, (float)kexp, (float)eps, (float)(1.0 / eps),
        (float)(kap * kap), coef, accumulate ? 1 : 0, out, sym ? c.d_symOff : nullptr,
        (const float2 *)c.d_symScr);
    return;
  }
  // the symmetric kernel for the context's own records (not the FP64 residual records of a mixed context)
  const bool sym = c.nSymTasks > 0 && tgtP == c.d_tgtP && (sizeof(T) == 8) == !c.mixed;
  if (sym) {
    near_pack_kernel<T><<<ceil_div(n, 256), 256, 0, s>>>(n, (const V *)tgtP, (const V *)tgtN, c.d_area, sgm,
                                                         (V *)c.d_symA, (V *)c.d_symB, 0);
    near_sym_kernel<T, ADJ><<<ceil_div(c.nSymTasks, kSymWarps), kSymWarps * 32, 0, s>>>(
        c.nSymTasks, c.d_symTask, c.d_leafStart, c.d_leafCount, c.d_leafCtr, (const V *)c.d_symA,
        (const V *)c.d_symB, (T)kap, (T)kexp, (T)eps, (T)(1.0 / eps), (T)(kap * kap), (T *)c.d_symScr);
    c.launches += 2;
  }
  near_apply_kernel<T, ADJ><<<grid, kNearWarps * 32, 0, s>>>(
      c.nWork, c.d_work, c.d_leafStart, c.d_leafCount, c.d_nearOff, c.d_nearSrc, c.d_leafCtr, (const V *)tgtP,
      (const V *)tgtN, (const V *)srcA, (const V *)srcB, c.d_spOff, c.d_spSrc, ADJ ? c.d_spKT : c.d_spK, sgm,
      c.d_area, n, (T)kap, (T)kexp, (T)eps, (T)(1.0 / eps), (T)(kap * kap), coef, accumulate ? 1 : 0, out,
      sym ? c.d_symOff : nullptr, (const T *)c.d_symScr);
}

// FP64 records in a mixed context, for the FP64 residuals of iterative
// refinement (built at context set-up)
static bool setup_near_fp64(Context &c) {
  if (c.d_tgtP64) return true;
  const int n = c.n;
  const size_t vb = sizeof(double4) * (size_t)n;
  if (!c.arena.alloc(&c.d_tgtP64, vb) || !c.arena.alloc(&c.d_tgtN64, vb) || !c.arena.alloc(&c.d_srcA64, vb) ||
      !c.arena.alloc(&c.d_srcB64, vb))
    return false;
  near_targets_kernel<double><<<ceil_div(n, 256), 256, 0, c.stream>>>(n, c.d_vtx, c.d_nrm, c.d_area, c.d_leafOfPanel,
                                                                      c.d_leafCtr, (double4 *)c.d_tgtP64,
                                                                      (double4 *)c.d_tgtN64);
  FB_CUDA(cudaGetLastError());
  return true;
}

// Transposed special-pair table: entry (X, Y) of row X holds the correction
// of the pair (Y, X) arranged for the ADJ epilogue
// (out_pot += dK3(Y,X) l_dpdn + dK1(Y,X) l_pot, out_dpdn += dK2(Y,X) l_dpdn + dK0(Y,X) l_pot).
__global__ void special_transpose_kernel(long long nSp, const long long *__restrict__ mate, const double4 *__restrict__ spK,
                                         double4 *spKT) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nSp) return;
  const double4 d = spK[mate[e]];
  spKT[e] = make_double4(d.w, d.y, d.z, d.x);
}

// mate[e] of entry e = (X, Y): the index of (Y, X); *bad = X + 1 when missing
__global__ void special_mate_kernel(int n, const int *__restrict__ spOff, const int *__restrict__ spSrc,
                                    long long *mate, int *bad) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  if (X >= n) return;
  for (int e = spOff[X]; e < spOff[X + 1]; e++) {
    const int Y = spSrc[e];
    int lo = spOff[Y], hi = spOff[Y + 1];
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (spSrc[mid] < X) lo = mid + 1;
      else hi = mid;
    }
    if (lo < spOff[Y + 1] && spSrc[lo] == X) mate[e] = lo;
    else atomicExch(bad, X + 1);
  }
}

static bool setup_near_adjoint(Context &c) {
  if (c.d_spKT) return true;
  // the special-pair set is symmetric (shared vertex, near leaf pairs): find
  // for every entry (X, Y) the entry (Y, X), by binary search in the
  // (ascending) row of Y, on the device
  const int n = c.n;
  DevArena tmp;
  long long *d_mate = nullptr;
  int *d_bad = nullptr;
  if (!tmp.alloc_n(&d_mate, (size_t)std::max<long long>(c.nSpecial, 1)) || !tmp.alloc_n(&d_bad, 1)) return false;
  FB_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), c.stream));
  special_mate_kernel<<<ceil_div(n, 256), 256, 0, c.stream>>>(n, c.d_spOff, c.d_spSrc, d_mate, d_bad);
  int bad = 0;
  FB_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  FB_CUDA(cudaStreamSynchronize(c.stream));
  FB_CHECK(bad == 0, "special pair (%d, .) has no mirror entry", bad - 1);
  if (!c.arena.alloc_n(&c.d_spKT, (size_t)std::max<long long>(c.nSpecial, 1))) return false;
  if (c.nSpecial > 0)
    special_transpose_kernel<<<ceil_div(c.nSpecial, 256), 256, 0, c.stream>>>(c.nSpecial, d_mate, c.d_spK, c.d_spKT);
  FB_CUDA(cudaGetLastError());
  FB_CUDA(cudaStreamSynchronize(c.stream));   // the mates are freed on return
  return true;
}

bool launch_near(Context &c, const double *sgm, double coef, double *out, bool adjoint, bool fp64,
                 cudaStream_t stream, bool accumulate) {
  if (adjoint && !setup_near_adjoint(c)) return false;
  cudaStream_t s = stream ? stream : c.stream;
  const bool acc = accumulate;
  if (c.prm.quad_order > 1) {   // every near pair by panelIA0 at order q, in FP64 in every context
    auto kern = adjoint ? near_quad_kernel<true> : near_quad_kernel<false>;
    kern<<<ceil_div(c.n, 128), 128, 0, s>>>(c.n, c.prm.quad_order, c.d_leafOfPanel, c.d_leafStart, c.d_leafCount,
                                            c.d_nearOff, c.d_nearSrc, c.d_vtx, c.d_nrm, c.d_area, c.prm.kappa,
                                            c.epsilon, sgm, coef, acc ? 1 : 0, out);
    c.launches += 1;
    FB_CUDA(cudaGetLastError());
    return true;
  }
  if (c.mixed && fp64) {
    if (!setup_near_fp64(c)) return false;
    if (adjoint) launch_near_t<double, true>(c, c.d_tgtP64, c.d_tgtN64, c.d_srcA64, c.d_srcB64, sgm, coef, out, s, acc);
    else launch_near_t<double, false>(c, c.d_tgtP64, c.d_tgtN64, c.d_srcA64, c.d_srcB64, sgm, coef, out, s, acc);
  } else if (c.mixed) {
    if (adjoint) launch_near_t<float, true>(c, c.d_tgtP, c.d_tgtN, c.d_srcA, c.d_srcB, sgm, coef, out, s, acc);
    else launch_near_t<float, false>(c, c.d_tgtP, c.d_tgtN, c.d_srcA, c.d_srcB, sgm, coef, out, s, acc);
  } else {
    if (adjoint) launch_near_t<double, true>(c, c.d_tgtP, c.d_tgtN, c.d_srcA, c.d_srcB, sgm, coef, out, s, acc);
    else launch_near_t<double, false>(c, c.d_tgtP, c.d_tgtN, c.d_srcA, c.d_srcB, sgm, coef, out, s, acc);
  }
  c.launches += 2;
  FB_CUDA(cudaGetLastError());
  return true;
}

}  // namespace fb
