// solver.cu -- preconditioner and restarted GMRES, resident on the device.
//
//   block preconditioner   src/precond_fmm.c:147-263, 553-652: one dense block
//                          per level (depth-1) cube, 2*nPnls square, entries
//                          block[i*M+j] from panelIA0(pnlX=j, pnlY=i) which
//                          LAPACK reads column-major, plus the area diagonal;
//                          LU-factored once (dgetrf)
//   cached-LU apply        src/precond_fmm.c:861-953 (dgetrs per block)
//   diagonal apply         src/precond_fmm.c:664-728
//   GMRES                  src/gmres.c:153-373 (Templates GMRES, left
//                          preconditioned, modified Gram-Schmidt basis,
//                          Givens rotations, x0 = initial guess)
//
// B200 design: the block matrices are assembled by a kernel in FP64 (the
// exact panelIA0 cases), factored with cuSOLVER at setup, and replaced by
// their explicit inverses, so each preconditioner apply is one block-diagonal
// GEMV kernel streaming the inverses from HBM instead of ~3 launches per
// block.  The Krylov vectors live on the device; the Gram-Schmidt dot
// products are reduced deterministically into a device array and only the
// (restart+1)-long Hessenberg column crosses to the host per iteration, where
// the Givens rotations run in FP64 exactly as in the reference.
#include <cusolverDn.h>

#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "context.cuh"
#include "quad.cuh"

namespace fb {

struct PrecondDev {
  int mode = -1;
  DevArena arena;
  int nBlocks = 0;
  std::vector<int> hStart, hSize;
  std::vector<long long> hOff;
  int *d_start = nullptr, *d_size = nullptr;
  int2 *d_tiles = nullptr;   // (block, first row) tiles of the apply
  int *d_colSrc = nullptr;   // per block (offset 2*start): input component of each stored column
  int nTiles = 0;
  long long *d_off = nullptr;
  double *d_inv = nullptr;
  float *d_invF = nullptr;   // mixed contexts: the inverses stored in FP32 (applied with FP64 sums)
  int maxM = 0;
  // GMRES workspace
  int restart = 0;
  double *d_V = nullptr, *d_r = nullptr, *d_av = nullptr, *d_w = nullptr;
  double *d_h = nullptr, *d_part = nullptr, *d_y = nullptr;
  double *d_H = nullptr, *d_sv = nullptr;   // Hessenberg (+ cs, sn columns) and rotated residual vector
  void *d_status = nullptr;                 // GmresStatus on the device
  void *h_status = nullptr;                 // pinned host copy (and two host-read norms)
  cudaEvent_t evStatus = nullptr;           // marks the status copy (the host spins on it)
  int partCap = 0;
};

void free_precond(Context &c) {
  if (c.pc) {
    c.pc->arena.release();
    if (c.pc->h_status) cudaFreeHost(c.pc->h_status);
    if (c.pc->evStatus) cudaEventDestroy(c.pc->evStatus);
    delete c.pc;
    c.pc = nullptr;
  }
}

// ---------------------------------------------------------------------------
// block assembly: A(j, i) = -K1(X=j,Y=i) etc. in column-major M x M
// (src/precond_fmm.c:147-263: panelIA0 over the cube's panel pairs).
// From the near field's own coefficients: every pair's one-point
// term A_X A_Y KER4(p_X - p_Y) at the one-point nodes p = v0/2 + v1/4 + v2/4 (0
// for X = Y), then, in pc_special_kernel, the exact-minus-one-point correction
// of the special pairs (shared vertex, edge, self) from the near field's table,
// so a block equals panelIA0's at -q=1 without its singularity tests per pair.
template <typename TO>
__global__ void pc_onepoint_kernel(int nBlocks, const int *__restrict__ bStart, const int *__restrict__ bSize,
                                   const long long *__restrict__ bOff, const double *__restrict__ vtx,
                                   const double *__restrict__ nrm, const double *__restrict__ area, double kappa,
                                   double eps, double s1, double s2, TO *A) {
  for (int b = blockIdx.y; b < nBlocks; b += gridDim.y) {   // (the grid's y extent is capped at 65535)
    const int hm = bSize[b], st = bStart[b], M = 2 * hm;
    const long long pairs = (long long)hm * hm;
    TO *Ab = A + bOff[b];
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < pairs;
         p += (long long)gridDim.x * blockDim.x) {
      const int i = (int)(p / hm), j = (int)(p % hm);  // i: pnlY (column), j: pnlX (row)
      const int Xi = st + j, Yi = st + i;
      double K[4] = {0.0, 0.0, 0.0, 0.0};
      if (Xi != Yi) {
        const double *vx = vtx + 9 * (size_t)Xi, *vy = vtx + 9 * (size_t)Yi;
        double r[3], nX[3], nY[3];
        for (int c = 0; c < 3; c++) {
          const double mx = vx[c] + 0.5 * ((vx[3 + c] - vx[c]) + 0.5 * (vx[6 + c] - vx[3 + c]));
          const double my = vy[c] + 0.5 * ((vy[3 + c] - vy[c]) + 0.5 * (vy[6 + c] - vy[3 + c]));
          r[c] = mx - my;
          nX[c] = nrm[3 * (size_t)Xi + c];
          nY[c] = nrm[3 * (size_t)Yi + c];
        }
        if (r[0] != 0.0 || r[1] != 0.0 || r[2] != 0.0) {
          double y[4];
          ker4_d(kappa, eps, r, nX, nY, y);
          const double w = area[Xi] * area[Yi];
          for (int k = 0; k < 4; k++) K[k] = w * y[k];
        }
      }
      const double d0 = (i == j) ? s1 * area[Yi] : 0.0;
      const double d1 = (i == j) ? s2 * area[Yi] : 0.0;
      Ab[(size_t)i * M + j] = (TO)(-K[1] + d0);
      Ab[(size_t)i * M + j + hm] = (TO)(-K[0]);
      Ab[(size_t)(i + hm) * M + j] = (TO)(-K[3]);
      Ab[(size_t)(i + hm) * M + j + hm] = (TO)(-K[2] + d1);
    }
  }
}

// the special pairs (X, Y) of a block: add their correction (each entry has one writer)
template <typename TO>
__global__ void pc_special_kernel(int nBlocks, const int *__restrict__ bStart, const int *__restrict__ bSize,
                                  const long long *__restrict__ bOff, const int *__restrict__ spOff,
                                  const int *__restrict__ spSrc, const double4 *__restrict__ spK, TO *A) {
  for (int b = blockIdx.y; b < nBlocks; b += gridDim.y) {
    const int hm = bSize[b], st = bStart[b], M = 2 * hm;
    TO *Ab = A + bOff[b];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < hm; j += gridDim.x * blockDim.x) {
      const int Xi = st + j;
      for (int e = spOff[Xi]; e < spOff[Xi + 1]; e++) {
        const int Yi = spSrc[e];
        if (Yi < st || Yi >= st + hm) continue;
        const int i = Yi - st;
        const double4 d = spK[e];   // (K0, K1, K2, K3) exact minus one-point
        TO *a0 = Ab + (size_t)i * M + j, *a1 = Ab + (size_t)i * M + j + hm;
        TO *a2 = Ab + (size_t)(i + hm) * M + j, *a3 = Ab + (size_t)(i + hm) * M + j + hm;
        *a0 = (TO)((double)*a0 - d.y);
        *a1 = (TO)((double)*a1 - d.x);
        *a2 = (TO)((double)*a2 - d.w);
        *a3 = (TO)((double)*a3 - d.z);
      }
    }
  }
}

// the listed blocks of I := identity, and their column index the identity
__global__ void identity_kernel(int nList, const int *__restrict__ list, const int *__restrict__ bStart,
                                const int *__restrict__ bSize, const long long *__restrict__ bOff, double *I,
                                int *colSrc) {
  for (int li = blockIdx.y; li < nList; li += gridDim.y) {   // (y extent capped at 65535)
    const int b = list[li];
    const int M = 2 * bSize[b];
    const long long e = (long long)M * M;
    double *Ib = I + bOff[b];
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < e; p += (long long)gridDim.x * blockDim.x)
      Ib[p] = ((p / M) == (p % M)) ? 1.0 : 0.0;
    if (blockIdx.x == 0)
      for (int c = threadIdx.x; c < M; c += blockDim.x) colSrc[2LL * bStart[b] + c] = c;
  }
}

// In-place inversion of the preconditioner blocks by blocked Gauss-Jordan
// elimination with partial (row) pivoting, all blocks in one launch per size
// class (a library LU costs tens of small launches per block).  A block is
// inverted by a cluster of CS thread blocks (CS = 1 for small blocks).  Per
// panel of NB columns:
//   * every CTA of the cluster eliminates the panel in its shared memory (the
//     same data, so the same result; pivot = first largest |a| at or below
//     the diagonal, as idamax) and rank 0 writes it back;
//   * each CTA takes its share of the other columns (64-column tiles dealt
//     round-robin): the panel's row interchanges, the panel rows moved to a
//     scratch Y and zeroed, then A(:, j) += Panel * Y(:, j), the composite
//     elimination of the panel as a rank-NB update (4x4 outputs per thread);
//   * a cluster barrier before the next panel, whose columns some CTA owns.
// The column interchanges that end Gauss-Jordan are not carried out:
// colSrc[c] records which input component stored column c multiplies, and
// the apply kernels gather through it.  info[b] = k+1 for an exactly zero
// pivot k.
constexpr int kGjThreads = 256;

template <typename TV, int NB>
__host__ __device__ constexpr size_t gj_smem_bytes(int maxM) {
  return (size_t)NB * maxM * sizeof(TV) + 64 * NB * sizeof(TV) + (size_t)maxM * sizeof(int);
}

// resident blocks per SM the register allocation of pc_gj_invert_kernel<float>
// aims at (the FP64 kernel keeps one: at two it spills)
#ifndef FB_GJ_MIN_BLOCKS
#define FB_GJ_MIN_BLOCKS 2
#endif
template <typename TV, int NB, int CS>
__global__ void __launch_bounds__(kGjThreads, sizeof(TV) == 4 ? FB_GJ_MIN_BLOCKS : 1)
pc_gj_invert_kernel(const int *__restrict__ list, const int *__restrict__ bStart, const int *__restrict__ bSize,
                    const long long *__restrict__ bOff, const long long *__restrict__ yOff, TV *inv, TV *yAll,
                    int *colSrc, int *info) {
  typedef typename Vec2<TV>::t V2;
  extern __shared__ double gjSmemD[];
  TV *gjSmem = reinterpret_cast<TV *>(gjSmemD);
  __shared__ TV wbest[kGjThreads / 32];
  __shared__ int wbi[kGjThreads / 32];
  __shared__ int sPos[2 * NB], sSrc[2 * NB], sCnt;
  __shared__ TV gBuf[64 * 2 * NB];   // one column tile's moved rows
  __shared__ TV sRk[NB], sOk[NB];
  const int rank = (CS > 1) ? (int)(blockIdx.x % CS) : 0;
  const int b = list[blockIdx.x / CS];
  const int M = 2 * bSize[b];
  TV *A = inv + bOff[b];
  TV *Y = yAll + yOff[b];
  TV *P = gjSmem;                          // panel, [NB][M]
  TV *Yt = gjSmem + (size_t)NB * M;        // Y tile, [64][NB]
  int *perm = (int *)(Yt + 64 * NB);           // [M]
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  int bad = 0;
  for (int k0 = 0; k0 < M; k0 += NB) {
    const int nb = min(NB, M - k0);
    if (CS > 1) {   // the owners' updates of these columns are complete and visible
      __threadfence();
      cooperative_groups::this_cluster().sync();
    }
    for (int e = t; e < nb * M; e += kGjThreads) P[e] = A[(size_t)k0 * M + e];   // columns k0.. are contiguous
    __syncthreads();
    // Row i of the panel belongs to thread i mod kGjThreads throughout: each
    // step's write phase also finds the thread's candidate pivot of the next
    // column among its own rows, so a step needs two barriers.
    TV best = (TV)-1;
    int bi = M;
    for (int i = t; i < M; i += kGjThreads) {
      if (i < k0) continue;
      const TV v = fabs(P[i]);
      if (v > best) { best = v; bi = i; }
    }
    for (int kk = 0; kk < nb; kk++) {
      const int k = k0 + kk;
      for (int o = 16; o > 0; o >>= 1) {   // first largest within the warp
        const TV ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) { wbest[warp] = best; wbi[warp] = bi; }
      __syncthreads();
      int pv = wbi[0];
      TV pb = wbest[0];
      for (int w = 1; w < kGjThreads / 32; w++)
        if (wbest[w] > pb || (wbest[w] == pb && wbi[w] < pv)) { pb = wbest[w]; pv = wbi[w]; }
      if (t == 0) perm[k] = pv;
      // read phase: the pivot row (old row pv, scaled; sRk[kk] = 1/pivot) and
      // the old row k, which moves to row pv
      if (t < nb) {
        const TV piv = P[kk * M + pv];
        const TV d = (piv != (TV)0) ? (TV)1 / piv : (TV)0;
        sRk[t] = (t == kk) ? d : P[t * M + pv] * d;
        sOk[t] = P[t * M + k];
      }
      if (P[kk * M + pv] == (TV)0) bad = bad ? bad : k + 1;
      __syncthreads();
      // write phase, and the candidates for the next column
      const TV d = sRk[kk];
      best = (TV)-1;
      bi = M;
      const bool more = kk + 1 < nb;
      for (int i = t; i < M; i += kGjThreads) {
        if (i == k) {
          for (int c = 0; c < nb; c++) P[c * M + k] = sRk[c];
          continue;   // the pivot row is no candidate
        }
        if (i == pv) {   // (only reached when pv != k) the old row k, eliminated
          const TV f = sOk[kk];
          for (int c = 0; c < nb; c++) P[c * M + i] = (c == kk) ? -f * d : sOk[c] - f * sRk[c];
        } else {
          const TV f = P[kk * M + i];
          for (int c = 0; c < nb; c++) P[c * M + i] = (c == kk) ? -f * d : P[c * M + i] - f * sRk[c];
        }
        if (more && i > k) {
          const TV v = fabs(P[(kk + 1) * M + i]);
          if (v > best) { best = v; bi = i; }
        }
      }
      // the next step's first barrier orders this write phase before its reads
    }
    __syncthreads();
    if (rank == 0)
      for (int e = t; e < nb * M; e += kGjThreads) A[(size_t)k0 * M + e] = P[e];
    // the panel's row interchanges as one gather: row r takes the value of row sSrc of the same column
    if (t == 0) {
      int cnt = 0;
      auto add = [&](int r) {
        for (int q = 0; q < cnt; q++)
          if (sPos[q] == r) return;
        sPos[cnt] = r;
        sSrc[cnt] = r;
        cnt++;
      };
      for (int kk = 0; kk < nb; kk++) {
        add(k0 + kk);
        add(perm[k0 + kk]);
      }
      for (int kk = 0; kk < nb; kk++) {   // replay the swaps on the source indices
        const int k = k0 + kk, pv = perm[k];
        int qa = 0, qb = 0;
        for (int q = 0; q < cnt; q++) {
          if (sPos[q] == k) qa = q;
          if (sPos[q] == pv) qb = q;
        }
        const int tmp = sSrc[qa];
        sSrc[qa] = sSrc[qb];
        sSrc[qb] = tmp;
      }
      sCnt = cnt;
    }
    __syncthreads();
    // this CTA's columns: gather the interchanged rows, rows k0.. to Y, zero
    // them; per 64-column tile all (column, moved row) reads are issued
    // together into gBuf, then, after a barrier, written back
    const int cnt = sCnt;
    for (int jt = 64 * rank; jt < M; jt += 64 * CS) {
      const int ne = 64 * cnt;
#pragma unroll 4
      for (int e = t; e < ne; e += kGjThreads) {
        const int jl = e / cnt, q = e - jl * cnt, j = jt + jl;
        if (j < M && (j < k0 || j >= k0 + nb)) gBuf[e] = A[(size_t)j * M + sSrc[q]];
      }
      __syncthreads();
      for (int e = t; e < ne; e += kGjThreads) {
        const int jl = e / cnt, q = e - jl * cnt, j = jt + jl;
        if (j < M && (j < k0 || j >= k0 + nb)) {
          const int r = sPos[q];
          TV *col = A + (size_t)j * M;
          if (r >= k0 && r < k0 + nb) {
            Y[(size_t)j * NB + (r - k0)] = gBuf[e];
            col[r] = (TV)0;
          } else {
            col[r] = gBuf[e];
          }
        }
      }
      __syncthreads();
    }
    // A(:, j) += P * Y(:, j) over this CTA's 64-column tiles; thread: 4 rows x 4 columns
    const int tr = t % 16, tc = t / 16;
    for (int jt = 64 * rank; jt < M; jt += 64 * CS) {
      for (int e = t; e < 64 * NB; e += kGjThreads) {
        const int jl = e / NB, kk = e % NB, j = jt + jl;
        const bool ok = j < M && (j < k0 || j >= k0 + nb) && kk < nb;
        Yt[e] = ok ? Y[(size_t)j * NB + kk] : (TV)0;
      }
      __syncthreads();
      // row tiles, the next tile's A values loaded while the current one is computed
      auto load_tile = [&](int it, TV (&v)[4][4]) {
        const int i0 = it + 4 * tr;
        const bool in = i0 < M, full = i0 + 4 <= M;   // M is even: a row quad is full or holds two rows
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int j = jt + 4 * tc + c;
          if (in && j < M) {
            const V2 *src = reinterpret_cast<const V2 *>(A + (size_t)j * M + i0);
            const V2 lo = src[0], hi = full ? src[1] : V2{(TV)0, (TV)0};
            v[c][0] = lo.x; v[c][1] = lo.y; v[c][2] = hi.x; v[c][3] = hi.y;
          } else {
            v[c][0] = v[c][1] = v[c][2] = v[c][3] = (TV)0;
          }
        }
      };
      TV acc[4][4], nxt[4][4];
      load_tile(0, acc);
      for (int it = 0; it < M; it += 64) {
        const int i0 = it + 4 * tr;
        if (it + 64 < M) load_tile(it + 64, nxt);
        if (i0 < M) {
          const bool full = i0 + 4 <= M;
          for (int kk = 0; kk < nb; kk++) {
            const V2 *pw = reinterpret_cast<const V2 *>(P + (size_t)kk * M + i0);
            const V2 wlo = pw[0], whi = full ? pw[1] : V2{(TV)0, (TV)0};
            const TV w[4] = {wlo.x, wlo.y, whi.x, whi.y};
            TV y[4];
#pragma unroll
            for (int c = 0; c < 4; c++) y[c] = Yt[(4 * tc + c) * NB + kk];
#pragma unroll
            for (int c = 0; c < 4; c++)
#pragma unroll
              for (int r = 0; r < 4; r++) acc[c][r] += w[r] * y[c];
          }
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int j = jt + 4 * tc + c;
            if (j < M && (j < k0 || j >= k0 + nb)) {
              V2 *dst = reinterpret_cast<V2 *>(A + (size_t)j * M + i0);
              dst[0] = V2{acc[c][0], acc[c][1]};
              if (full) dst[1] = V2{acc[c][2], acc[c][3]};
            }
          }
        }
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
          for (int r = 0; r < 4; r++) acc[c][r] = nxt[c][r];
      }
      __syncthreads();
    }
  }
  // the pending column interchanges, as an index: stored column c multiplies input component colSrc[c]
  __syncthreads();
  if (rank == 0 && t == 0) {
    // sigma: final column j = stored column sigma[j], built by replaying the swaps in reverse
    int *cs = colSrc + 2 * bStart[b];
    for (int c = 0; c < M; c++) cs[c] = c;   // cs temporarily holds sigma
    for (int k = M - 1; k >= 0; k--) {
      const int pv = perm[k];
      if (pv != k) {
        const int a = cs[k];
        cs[k] = cs[pv];
        cs[pv] = a;
      }
    }
    // invert: colSrc[sigma[j]] = j
    for (int j = 0; j < M; j++) perm[cs[j]] = j;
    for (int c = 0; c < M; c++) cs[c] = perm[c];
    info[b] = bad;
  }
  if (CS > 1) cooperative_groups::this_cluster().sync();   // no CTA leaves while others may still read
}

// x = blockdiag(inv) * b, block b gathers its pot/dpdn halves
// Block-diagonal apply with the explicit inverses, one thread block per tile
// of kPcRows rows of one diagonal block (tiles of large blocks spread over
// many SMs).  The block's inputs are gathered into shared memory (in chunks
// of kPcChunk columns); warp w sums the columns c = w mod kPcWarps, each lane
// kPcRpl consecutive rows (8- or 16-byte loads of the column-major inverse,
// eight columns in flight), and the warps' partial sums are added in a fixed
// order.  The reference's per-block solve order (x = [pot; dpdn]
// of the cube's panels) is src/precond_fmm.c:861-953.
#ifndef FB_PC_RPL
#define FB_PC_RPL 4
#endif
constexpr int kPcRpl = FB_PC_RPL;   // rows per lane (2 or 4)
constexpr int kPcRows = 32 * kPcRpl, kPcWarps = 8, kPcChunk = 2048;

// streams the block factorisations are spread over
#ifndef FB_PC_STREAMS
#define FB_PC_STREAMS 16
#endif

template <typename TI>
__global__ void __launch_bounds__(kPcWarps * 32)
pc_apply_kernel(int n, const int2 *__restrict__ tiles, const int *__restrict__ bStart, const int *__restrict__ bSize,
                const long long *__restrict__ bOff, const int *__restrict__ colSrc, const TI *__restrict__ inv,
                const double *__restrict__ rhs, double *x) {
  typedef typename Vec2<TI>::t V2;
  __shared__ double xs[kPcChunk];
  __shared__ double red[kPcWarps][kPcRows];
  const int2 tl = tiles[blockIdx.x];
  const int b = tl.x, r0 = tl.y;
  const int hm = bSize[b], st = bStart[b], M = 2 * hm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = r0 + kPcRpl * lane;   // M is even: rows r and r + 1 are both in or both out
  const TI *Ib = inv + bOff[b];
  const int *cs = colSrc + 2 * (size_t)st;
  double y0 = 0.0, y1 = 0.0, y2 = 0.0, y3 = 0.0;
  const bool q2 = kPcRpl == 4 && r + 2 < M;
  for (int k0 = 0; k0 < M; k0 += kPcChunk) {
    const int kn = min(kPcChunk, M - k0);
    __syncthreads();   // the previous chunk's reads are done
    for (int c = threadIdx.x; c < kn; c += blockDim.x) {
      const int g = cs[k0 + c];
      xs[c] = (g < hm) ? rhs[st + g] : rhs[n + st + g - hm];
    }
    __syncthreads();
    if (r < M) {
      const TI *col = Ib + (size_t)k0 * M + r;
#pragma unroll 8
      for (int c = warp; c < kn; c += kPcWarps) {
        const V2 a = *reinterpret_cast<const V2 *>(col + (size_t)c * M);
        const double xc = xs[c];
        y0 += (double)a.x * xc;
        y1 += (double)a.y * xc;
        if (kPcRpl == 4 && q2) {
          const V2 a2 = *reinterpret_cast<const V2 *>(col + (size_t)c * M + 2);
          y2 += (double)a2.x * xc;
          y3 += (double)a2.y * xc;
        }
      }
    }
  }
  red[warp][kPcRpl * lane] = y0;
  red[warp][kPcRpl * lane + 1] = y1;
  if (kPcRpl == 4) {
    red[warp][kPcRpl * lane + 2] = y2;
    red[warp][kPcRpl * lane + 3] = y3;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kPcRows; i += blockDim.x) {
    const int rr = r0 + i;
    if (rr < M) {
      double t = red[0][i];
#pragma unroll
      for (int w = 1; w < kPcWarps; w++) t += red[w][i];
      if (rr < hm) x[st + rr] = t;
      else x[n + st + rr - hm] = t;
    }
  }
}

// Transposed block-diagonal apply (adjoint solves): output c of a block is
// column c of its inverse dotted with the block's input.  Tiles of kPcRows
// outputs; the block's input is staged in shared memory in chunks, a warp per
// output column, each lane two consecutive rows per step.
template <typename TI>
__global__ void __launch_bounds__(kPcWarps * 32)
pc_apply_t_kernel(int n, const int2 *__restrict__ tiles, const int *__restrict__ bStart, const int *__restrict__ bSize,
                  const long long *__restrict__ bOff, const int *__restrict__ colSrc, const TI *__restrict__ inv,
                  const double *__restrict__ rhs, double *x) {
  typedef typename Vec2<TI>::t V2;
  __shared__ double xs[kPcChunk];
  const int2 tl = tiles[blockIdx.x];
  const int b = tl.x, c0 = tl.y;
  const int hm = bSize[b], st = bStart[b], M = 2 * hm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const TI *Ib = inv + bOff[b];
  constexpr int kCols = kPcRows / kPcWarps;   // output columns per warp
  double y[kCols];
#pragma unroll
  for (int q = 0; q < kCols; q++) y[q] = 0.0;
  for (int k0 = 0; k0 < M; k0 += kPcChunk) {
    const int kn = min(kPcChunk, M - k0);
    __syncthreads();
    for (int i = threadIdx.x; i < kn; i += blockDim.x) {
      const int rr = k0 + i;
      xs[i] = (rr < hm) ? rhs[st + rr] : rhs[n + st + rr - hm];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kCols; q++) {
      const int c = c0 + warp + q * kPcWarps;
      if (c < M) {
        const TI *col = Ib + (size_t)c * M + k0;
        double acc = 0.0;
#pragma unroll 4
        for (int i = 2 * lane; i < kn; i += 64) {   // kn is even
          const V2 a = *reinterpret_cast<const V2 *>(col + i);
          acc += (double)a.x * xs[i] + (double)a.y * xs[i + 1];
        }
        y[q] += acc;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kCols; q++) {
    double v = y[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int c = c0 + warp + q * kPcWarps;
    if (lane == 0 && c < M) {
      const int g = colSrc[2 * (size_t)st + c];   // stored column c is output component g
      if (g < hm) x[st + g] = v;
      else x[n + st + g - hm] = v;
    }
  }
}

__global__ void pc_diag_kernel(int n, const double *__restrict__ area, double s1, double s2,
                               const double *__restrict__ b, double *x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = b[i] / (s1 * area[i]);
  x[n + i] = b[n + i] / (s2 * area[i]);
}

// LU and explicit inverse of every block with cuSOLVER (blocks above the
// Gauss-Jordan kernel's size limit), spread over several streams so that
// independent blocks run side by side.  Inverts d_A into p.d_inv.
static bool factor_cusolver(Context &c, PrecondDev &p, const std::vector<int> &blocks) {
  cudaStream_t s = c.stream;
  if (blocks.empty()) return true;
  // copy the assembled blocks out of d_inv, which then starts as the identity
  std::vector<long long> aOff(p.nBlocks, -1);
  long long atot = 0;
  int maxM = 0;
  for (int b : blocks) {
    aOff[b] = atot;
    atot += 4LL * p.hSize[b] * p.hSize[b];
    maxM = std::max(maxM, 2 * p.hSize[b]);
  }
  double *d_A = nullptr;
  FB_CUDA(cudaMalloc((void **)&d_A, (size_t)atot * sizeof(double)));
  for (int b : blocks)
    FB_CUDA(cudaMemcpyAsync(d_A + aOff[b], p.d_inv + p.hOff[b], 4LL * p.hSize[b] * p.hSize[b] * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
  const int ns = std::min(FB_PC_STREAMS, std::max((int)blocks.size(), 1));
  std::vector<cusolverDnHandle_t> hs(ns, nullptr);
  std::vector<cudaStream_t> ss(ns, nullptr);
  std::vector<double *> works(ns, nullptr);
  std::vector<int *> pivs(ns, nullptr);
  int lwork = 0, *d_info = nullptr;
  int *d_list = nullptr;
  FB_CUDA(cudaMalloc((void **)&d_list, blocks.size() * sizeof(int)));
  FB_CUDA(cudaMemcpyAsync(d_list, blocks.data(), blocks.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  dim3 grid(64, (unsigned)std::min<size_t>(blocks.size(), 65535));
  identity_kernel<<<grid, 256, 0, s>>>((int)blocks.size(), d_list, p.d_start, p.d_size, p.d_off, p.d_inv, p.d_colSrc);
  cudaEvent_t evA = nullptr;
  bool ok = cudaEventCreateWithFlags(&evA, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaEventRecord(evA, s) == cudaSuccess;
  for (int k = 0; ok && k < ns; k++) {
    ok = cudaStreamCreateWithFlags(&ss[k], cudaStreamNonBlocking) == cudaSuccess &&
         cusolverDnCreate(&hs[k]) == CUSOLVER_STATUS_SUCCESS && cusolverDnSetStream(hs[k], ss[k]) == CUSOLVER_STATUS_SUCCESS &&
         cudaStreamWaitEvent(ss[k], evA, 0) == cudaSuccess;
  }
  if (ok && cusolverDnDgetrf_bufferSize(hs[0], maxM, maxM, d_A, maxM, &lwork) != CUSOLVER_STATUS_SUCCESS) ok = false;
  for (int k = 0; ok && k < ns; k++)
    ok = cudaMalloc((void **)&works[k], (size_t)std::max(lwork, 1) * sizeof(double)) == cudaSuccess &&
         cudaMalloc((void **)&pivs[k], (size_t)maxM * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc((void **)&d_info, (size_t)p.nBlocks * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMemsetAsync(d_info, 0, (size_t)p.nBlocks * sizeof(int), s) == cudaSuccess;
  std::vector<int> order(blocks);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p.hSize[a] > p.hSize[b]; });
  for (int q = 0; ok && q < (int)order.size(); q++) {
    const int b = order[q], k = q % ns;
    int M = 2 * p.hSize[b];
    if (M == 0) continue;
    double *Ab = d_A + aOff[b], *Ib = p.d_inv + p.hOff[b];
    if (cusolverDnDgetrf(hs[k], M, M, Ab, M, works[k], pivs[k], d_info + b) != CUSOLVER_STATUS_SUCCESS) ok = false;
    if (ok && cusolverDnDgetrs(hs[k], CUBLAS_OP_N, M, M, Ab, M, pivs[k], Ib, M, d_info + b) != CUSOLVER_STATUS_SUCCESS)
      ok = false;
  }
  for (int k = 0; k < ns; k++) {
    if (!ss[k]) continue;
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(ev, ss[k]);
      cudaStreamWaitEvent(s, ev, 0);
      cudaEventDestroy(ev);
    } else {
      ok = false;
    }
  }
  std::vector<int> info(p.nBlocks, 0);
  if (ok) ok = cudaMemcpyAsync(info.data(), d_info, info.size() * sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess;
  if (ok) ok = cudaStreamSynchronize(s) == cudaSuccess;
  for (int k = 0; k < ns; k++) {
    if (ss[k]) cudaStreamSynchronize(ss[k]);
    if (hs[k]) cusolverDnDestroy(hs[k]);
    if (ss[k]) cudaStreamDestroy(ss[k]);
    cudaFree(works[k]);
    cudaFree(pivs[k]);
  }
  if (evA) cudaEventDestroy(evA);
  cudaFree(d_info);
  cudaFree(d_list);
  cudaFree(d_A);
  FB_CHECK(ok, "preconditioner factorisation failed: %s", cudaGetErrorString(cudaGetLastError()));
  for (int b = 0; b < p.nBlocks; b++)
    FB_CHECK(info[b] == 0, "dgetrf failed in preconditioner block %d (info=%d)", b, info[b]);
  return true;
}

// Blocks up to this many rows (and up to the size classes below) go to the
// Gauss-Jordan kernel; larger ones to cuSOLVER (several streams, FP64 only).
// Measured on the 204,800-panel star surface, sending everything to the
// kernel is fastest (cuSOLVER launches run slowly beside the kernel's
// resident blocks).
#ifndef FB_PC_GJ_MAXM
#define FB_PC_GJ_MAXM 11000
#endif
// CTAs per block for blocks of 385-768 rows (1 or 2; larger blocks use 8)
#ifndef FB_PC_GJ_MIDCS
#define FB_PC_GJ_MIDCS 2
#endif

template <typename TV, int NB, int CS>
static bool launch_gj_t(int nList, int maxM, cudaStream_t st, const int *d_list, PrecondDev &p, const long long *d_yOff,
                        TV *inv, TV *d_y, int *d_info) {
  const size_t shm = gj_smem_bytes<TV, NB>(maxM);
  cudaFuncAttributes fa{};
  FB_CUDA(cudaFuncGetAttributes(&fa, pc_gj_invert_kernel<TV, NB, CS>));
  int dev = 0, optin = 0;
  FB_CUDA(cudaGetDevice(&dev));
  FB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  FB_CHECK(shm + fa.sharedSizeBytes <= (size_t)optin,
           "Gauss-Jordan class NB=%d: %d rows need %zu + %zu bytes of shared memory, above the %d available", NB,
           maxM, shm, (size_t)fa.sharedSizeBytes, optin);
  FB_CUDA(cudaFuncSetAttribute(pc_gj_invert_kernel<TV, NB, CS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)shm));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nList * CS));
  cfg.blockDim = dim3(kGjThreads);
  cfg.dynamicSmemBytes = shm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  FB_CUDA(cudaLaunchKernelEx(&cfg, pc_gj_invert_kernel<TV, NB, CS>, d_list, (const int *)p.d_start,
                             (const int *)p.d_size, (const long long *)p.d_off, d_yOff, inv, d_y, p.d_colSrc,
                             d_info));
  return true;
}

template <typename TV>
static bool launch_gj(int nb, int cs, int nList, int maxM, cudaStream_t st, const int *d_list, PrecondDev &p,
                      const long long *d_yOff, TV *inv, TV *d_y, int *d_info) {
  if (nb == 16 && cs == 1) return launch_gj_t<TV, 16, 1>(nList, maxM, st, d_list, p, d_yOff, inv, d_y, d_info);
  if (nb == 16 && cs == 2) return launch_gj_t<TV, 16, 2>(nList, maxM, st, d_list, p, d_yOff, inv, d_y, d_info);
  if (nb == 16 && cs == 8) return launch_gj_t<TV, 16, 8>(nList, maxM, st, d_list, p, d_yOff, inv, d_y, d_info);
  if (nb == 8 && cs == 8) return launch_gj_t<TV, 8, 8>(nList, maxM, st, d_list, p, d_yOff, inv, d_y, d_info);
  if constexpr (sizeof(TV) == 4) return launch_gj_t<TV, 4, 8>(nList, maxM, st, d_list, p, d_yOff, inv, d_y, d_info);
  set_error("no Gauss-Jordan class with panel width %d", nb);
  return false;
}

// Size classes of the Gauss-Jordan kernel per precision: rows up to, panel
// width NB, CTAs per block (the panel of NB columns and the pivot record fit
// in shared memory).  Blocks above the last class go to cuSOLVER (FP64).
struct GjCls { int hi, nb, cs; };
template <typename TV>
static const GjCls *gj_classes(int *count) {
  // FP64 stops at 3200 rows: above it cuSOLVER's factorisation of a single
  // large block (all SMs) beats the kernel's narrow panels (measured on a
  // 2.1M-panel surface: 7.9 s against 9.8 s for the whole inversion)
  // (the NB = 16 FP64 panel of 1536 rows plus the kernel's static shared
  // memory is the largest that fits in the 227 KiB a block may use)
  static const GjCls d64[4] = {{384, 16, 1}, {768, 16, FB_PC_GJ_MIDCS}, {1536, 16, 8}, {3200, 8, 8}};
  static const GjCls d32[5] = {{384, 16, 1}, {768, 16, FB_PC_GJ_MIDCS}, {3200, 16, 8}, {6000, 8, 8}, {11000, 4, 8}};
  *count = sizeof(TV) == 8 ? 4 : 5;
  return sizeof(TV) == 8 ? d64 : d32;
}

template <typename TV>
static int gj_max_rows() {
  int n = 0;
  const GjCls *c = gj_classes<TV>(&n);
  return std::min(c[n - 1].hi, FB_PC_GJ_MAXM);
}

// Gauss-Jordan inversion of every block of inv (assembled there), size
// classes on their own streams so the large blocks start at once; blocks
// above the kernel's size limit (FP64 only) go to cuSOLVER meanwhile.
template <typename TV>
static bool factor_gauss_jordan(Context &c, PrecondDev &p, TV *inv) {
  cudaStream_t s = c.stream;
  const int cut = gj_max_rows<TV>();
  int ncls = 0;
  const GjCls *cls = gj_classes<TV>(&ncls);
  std::vector<int> big;
  for (int b = 0; b < p.nBlocks; b++)
    if (2 * p.hSize[b] > cut) big.push_back(b);
  FB_CHECK(big.empty() || sizeof(TV) == 8, "preconditioner block of %d rows above the FP32 limit %d", p.maxM, cut);
  std::vector<long long> yOff(p.nBlocks);
  long long ytot = 0;
  for (int b = 0; b < p.nBlocks; b++) {
    yOff[b] = ytot;
    ytot += 16LL * 2 * p.hSize[b];
  }
  long long *d_yOff = nullptr;
  TV *d_y = nullptr;
  int *d_info = nullptr;
  DevArena tmp;
  if (!tmp.upload(&d_yOff, yOff, s) || !tmp.alloc_n(&d_y, (size_t)std::max(ytot, 1LL)) ||
      !tmp.alloc_n(&d_info, (size_t)p.nBlocks))
    return false;
  FB_CUDA(cudaMemsetAsync(d_info, 0, (size_t)p.nBlocks * sizeof(int), s));
  cudaEvent_t evA = nullptr;
  FB_CUDA(cudaEventCreateWithFlags(&evA, cudaEventDisableTiming));
  FB_CUDA(cudaEventRecord(evA, s));
  std::vector<cudaStream_t> ss;
  bool ok = true;
  for (int ci = 0; ci < ncls; ci++) {
    const GjCls &k = cls[ci];
    const int lo = ci ? cls[ci - 1].hi : 0, hi = std::min(k.hi, cut);
    std::vector<int> list;
    int maxM = 0;
    for (int b = 0; b < p.nBlocks; b++) {
      const int M = 2 * p.hSize[b];
      if (hi > lo && M > lo && M <= hi) {
        list.push_back(b);
        maxM = std::max(maxM, M);
      }
    }
    if (list.empty()) continue;
    std::stable_sort(list.begin(), list.end(), [&](int a, int b) { return p.hSize[a] > p.hSize[b]; });
    int *d_list = nullptr;
    cudaStream_t st = nullptr;
    ok = ok && tmp.upload(&d_list, list, s) && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) break;
    ss.push_back(st);
    cudaEvent_t evL = nullptr;   // the list upload and the assembly on s come first
    ok = cudaEventCreateWithFlags(&evL, cudaEventDisableTiming) == cudaSuccess && cudaEventRecord(evL, s) == cudaSuccess &&
         cudaStreamWaitEvent(st, evL, 0) == cudaSuccess;
    if (evL) cudaEventDestroy(evL);
    if (!ok) break;
    if (!launch_gj<TV>(k.nb, k.cs, (int)list.size(), maxM, st, d_list, p, d_yOff, inv, d_y, d_info)) {
      ok = false;
      break;
    }
    c.launches += 1;
    ok = cudaGetLastError() == cudaSuccess;
  }
  // the large blocks meanwhile, through cuSOLVER on its own streams
  if (ok && !big.empty()) {
    if constexpr (sizeof(TV) == 8) ok = factor_cusolver(c, p, big);
  }
  for (cudaStream_t st : ss) {
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(ev, st);
      cudaStreamWaitEvent(s, ev, 0);
      cudaEventDestroy(ev);
    }
  }
  std::vector<int> info(p.nBlocks, 0);
  if (ok) ok = cudaMemcpyAsync(info.data(), d_info, info.size() * sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess;
  if (ok) ok = cudaStreamSynchronize(s) == cudaSuccess;
  for (cudaStream_t st : ss) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  cudaEventDestroy(evA);
  tmp.release();
  FB_CHECK(ok, "preconditioner inversion failed: %s", cudaGetErrorString(cudaGetLastError()));
  for (int b = 0; b < p.nBlocks; b++)
    FB_CHECK(info[b] == 0, "zero pivot in preconditioner block %d (step %d)", b, info[b]);
  return true;
}

bool precond_setup(Context &c, int mode) {
  free_precond(c);
  c.pc = new PrecondDev();
  PrecondDev &p = *c.pc;
  p.mode = mode;
  if (mode != 2) return true;   // -1 identity and 3 diagonal need no setup
  const Octree &t = c.pt.t;
  const int lev = t.depth - 1;
  FB_CHECK(lev >= 0, "block preconditioner needs depth >= 1");
  long long off = 0;
  for (int cc = t.levStart[lev]; cc < t.levStart[lev + 1]; cc++) {
    int hm = t.itemCount[cc];
    p.hStart.push_back(t.itemStart[cc]);
    p.hSize.push_back(hm);
    p.hOff.push_back(off);
    off += 4LL * hm * hm;
    p.maxM = std::max(p.maxM, 2 * hm);
  }
  p.nBlocks = (int)p.hSize.size();
  // apply tiles, the largest blocks' first (a tile's cost grows with its block's size)
  std::vector<int> order(p.nBlocks);
  for (int b = 0; b < p.nBlocks; b++) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p.hSize[a] > p.hSize[b]; });
  std::vector<int2> tiles;
  for (int b : order)
    for (int r0 = 0; r0 < 2 * p.hSize[b]; r0 += kPcRows) tiles.push_back(make_int2(b, r0));
  p.nTiles = (int)tiles.size();
  FB_CHECK(p.maxM <= 46340, "preconditioner block %d too large (increase -t)", p.maxM);
  cudaStream_t s = c.stream;
  StageTimer tm("precond_setup", s);
  if (!p.arena.upload(&p.d_start, p.hStart, s) || !p.arena.upload(&p.d_size, p.hSize, s) ||
      !p.arena.upload(&p.d_tiles, tiles, s) || !p.arena.upload(&p.d_off, p.hOff, s) ||
      !p.arena.alloc_n(&p.d_colSrc, 2 * (size_t)c.n))
    return false;
  // FP64 contexts invert in FP64; mixed contexts assemble and invert in FP32
  // (the preconditioner only steers GMRES; its inverse is stored in FP32)
  const double s1 = (1.0 + c.epsilon) / 2.0, s2 = (1.0 + 1.0 / c.epsilon) / 2.0;
  dim3 grid(64, std::min(p.nBlocks, 65535));
  bool ok;
  if (c.mixed) {
    FB_CHECK(p.maxM <= gj_max_rows<float>(), "preconditioner block of %d rows above the FP32 limit %d", p.maxM,
             gj_max_rows<float>());
    if (!p.arena.alloc_n(&p.d_invF, (size_t)off)) return false;
    pc_onepoint_kernel<float><<<grid, 128, 0, s>>>(p.nBlocks, p.d_start, p.d_size, p.d_off, c.d_vtx, c.d_nrm,
                                                   c.d_area, c.prm.kappa, c.epsilon, s1, s2, p.d_invF);
    pc_special_kernel<float><<<dim3(4, grid.y), 128, 0, s>>>(p.nBlocks, p.d_start, p.d_size, p.d_off, c.d_spOff,
                                                             c.d_spSrc, c.d_spK, p.d_invF);
    c.launches += 2;
    FB_CUDA(cudaGetLastError());
    tm.mark("assemble");
    ok = factor_gauss_jordan<float>(c, p, p.d_invF);
  } else {
    if (!p.arena.alloc_n(&p.d_inv, (size_t)off)) return false;
    pc_onepoint_kernel<double><<<grid, 128, 0, s>>>(p.nBlocks, p.d_start, p.d_size, p.d_off, c.d_vtx, c.d_nrm,
                                                    c.d_area, c.prm.kappa, c.epsilon, s1, s2, p.d_inv);
    pc_special_kernel<double><<<dim3(4, grid.y), 128, 0, s>>>(p.nBlocks, p.d_start, p.d_size, p.d_off, c.d_spOff,
                                                              c.d_spSrc, c.d_spK, p.d_inv);
    c.launches += 2;
    FB_CUDA(cudaGetLastError());
    tm.mark("assemble");
    ok = factor_gauss_jordan<double>(c, p, p.d_inv);
  }
  tm.mark("factor_invert");
  return ok;
}

bool precond_apply(Context &c, const double *b, double *x, bool adjoint) {
  FB_CHECK(c.pc != nullptr, "preconditioner not set up");
  PrecondDev &p = *c.pc;
  if (p.mode == 2 && adjoint) {
    if (p.d_invF)
      pc_apply_t_kernel<float><<<p.nTiles, kPcWarps * 32, 0, c.stream>>>(c.n, p.d_tiles, p.d_start, p.d_size,
                                                                             p.d_off, p.d_colSrc, p.d_invF, b, x);
    else
      pc_apply_t_kernel<double><<<p.nTiles, kPcWarps * 32, 0, c.stream>>>(c.n, p.d_tiles, p.d_start, p.d_size,
                                                                              p.d_off, p.d_colSrc, p.d_inv, b, x);
  } else if (p.mode == 2) {
    if (p.d_invF)
      pc_apply_kernel<float><<<p.nTiles, kPcWarps * 32, 0, c.stream>>>(c.n, p.d_tiles, p.d_start, p.d_size,
                                                                           p.d_off, p.d_colSrc, p.d_invF, b, x);
    else
      pc_apply_kernel<double><<<p.nTiles, kPcWarps * 32, 0, c.stream>>>(c.n, p.d_tiles, p.d_start, p.d_size,
                                                                             p.d_off, p.d_colSrc, p.d_inv, b, x);
  } else if (p.mode == 3) {
    pc_diag_kernel<<<ceil_div(c.n, 256), 256, 0, c.stream>>>(c.n, c.d_area, (1.0 + c.epsilon) / 2.0,
                                                            (1.0 + 1.0 / c.epsilon) / 2.0, b, x);
  } else {
    FB_CUDA(cudaMemcpyAsync(x, b, 2 * (size_t)c.n * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    return true;
  }
  c.launches += 1;
  FB_CUDA(cudaGetLastError());
  return true;
}

// ---------------------------------------------------------------------------
// level-1 kernels with deterministic reductions
// ---------------------------------------------------------------------------
constexpr int kRedBlocks = 296;   // 2 x 148 SMs
constexpr int kRedThreads = 256;

// part[b] = sum over the block's grid-stride share of x.*y
__global__ void dot_partial_kernel(long long n, const double *__restrict__ x, const double *__restrict__ y,
                                   double *part) {
  __shared__ double red[kRedThreads];
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// out[0] = sum(part) (or sqrt of it), fixed order
__global__ void dot_final_kernel(int k, const double *__restrict__ part, double *out, int takeSqrt) {
  __shared__ double red[kRedThreads];
  double s = 0.0;
  for (int i = threadIdx.x; i < k; i += blockDim.x) s += part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int m = blockDim.x / 2; m > 0; m >>= 1) {
    if ((int)threadIdx.x < m) red[threadIdx.x] += red[threadIdx.x + m];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = takeSqrt ? sqrt(red[0]) : red[0];
}

// y -= (*h) * x
__global__ void axpy_neg_dev_kernel(long long n, const double *__restrict__ h, const double *__restrict__ x, double *y) {
  const double a = -(*h);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

// v = w / (*h) when *h > 0, else v = w
__global__ void scale_copy_dev_kernel(long long n, const double *__restrict__ h, const double *__restrict__ w, double *v) {
  const double d = *h;
  const double s = (d > 0.0) ? 1.0 / d : 1.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = (d > 0.0) ? w[i] * s : w[i];
}

__global__ void scale_copy_kernel(long long n, double s, const double *__restrict__ w, double *v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = w[i] * s;
}

// x += V y  (k columns of length n, column stride ldv)
__global__ void update_kernel(long long n, int k, const double *__restrict__ V, long long ldv,
                              const double *__restrict__ y, double *x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = x[i];
    for (int j = 0; j < k; j++) s += y[j] * V[(size_t)j * ldv + i];
    x[i] = s;
  }
}

// Sum of kRedBlocks partials in a fixed order (the dot_final_kernel order),
// by every thread block alike; returns the total to all threads.
__device__ __forceinline__ double block_sum_partials(const double *__restrict__ part, double *red) {
  double s = 0.0;
  for (int i = threadIdx.x; i < kRedBlocks; i += blockDim.x) s += part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int m = blockDim.x / 2; m > 0; m >>= 1) {
    if ((int)threadIdx.x < m) red[threadIdx.x] += red[threadIdx.x + m];
    __syncthreads();
  }
  const double t = red[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ void block_store_partial(double acc, double *red, double *partOut) {
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int m = blockDim.x / 2; m > 0; m >>= 1) {
    if ((int)threadIdx.x < m) red[threadIdx.x] += red[threadIdx.x + m];
    __syncthreads();
  }
  if (threadIdx.x == 0) partOut[blockIdx.x] = red[0];
}

// One modified Gram-Schmidt column (gmres.c's ddot + daxpy pair) as a single
// launch on kRedBlocks blocks: every block reduces the partials of
// h_k = w.v_k in the same order, block 0 stores h_k, each block updates its
// grid-stride share w -= h_k v_k and leaves its partial of the next product,
// w.v_next (or w.w when v_next is null).  The grid partition is that of
// dot_partial_kernel, so the values equal the separate dot/axpy sequence.
__global__ void __launch_bounds__(kRedThreads)
mgs_step_kernel(long long n, const double *__restrict__ partIn, double *hk, const double *__restrict__ vk,
                const double *__restrict__ vnext, double *w, double *partOut) {
  __shared__ double red[kRedThreads];
  const double h = block_sum_partials(partIn, red);
  if (blockIdx.x == 0 && threadIdx.x == 0) *hk = h;
  const double a = -h;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double wi = w[i] + a * vk[i];
    w[i] = wi;
    acc += wi * (vnext ? vnext[i] : wi);
  }
  block_store_partial(acc, red, partOut);
}

// h_i = sqrt(w.w) from the partials; v_i = w / h_i (w itself when h_i is 0)
__global__ void __launch_bounds__(kRedThreads)
mgs_norm_scale_kernel(long long n, const double *__restrict__ partIn, double *hi, const double *__restrict__ w,
                      double *v) {
  __shared__ double red[kRedThreads];
  const double d = sqrt(block_sum_partials(partIn, red));
  if (blockIdx.x == 0 && threadIdx.x == 0) *hi = d;
  const double sc = (d > 0.0) ? 1.0 / d : 1.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = (d > 0.0) ? w[i] * sc : w[i];
}

static bool dot_dev(Context &c, long long n, const double *x, const double *y, double *out, bool sq) {
  PrecondDev &p = *c.pc;
  dot_partial_kernel<<<kRedBlocks, kRedThreads, 0, c.stream>>>(n, x, y, p.d_part);
  dot_final_kernel<<<1, kRedThreads, 0, c.stream>>>(kRedBlocks, p.d_part, out, sq ? 1 : 0);
  c.launches += 2;
  FB_CUDA(cudaGetLastError());
  return true;
}

// x . y to the host (fixed-order reduction); needs a preconditioner record
// for its scratch
bool dot_to_host(Context &c, long long n, const double *x, const double *y, double *out) {
  FB_CHECK(c.pc != nullptr, "dot_to_host without a preconditioner record");
  PrecondDev &p = *c.pc;
  if (!p.d_part && !p.arena.alloc_n(&p.d_part, 2 * (size_t)kRedBlocks + 2)) return false;
  if (!dot_dev(c, n, x, y, p.d_part + kRedBlocks, false)) return false;
  FB_CUDA(cudaMemcpyAsync(out, p.d_part + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  FB_CUDA(cudaStreamSynchronize(c.stream));
  return true;
}

// ---------------------------------------------------------------------------
// GMRES state on the device.  The Hessenberg matrix, the Givens rotations
// (cs, sn), the rotated residual vector s and the residual estimate live in
// device memory; one single-warp kernel per Arnoldi step applies the previous
// rotations to the new column, forms the next rotation (netlib drotg, the
// BLAS the reference calls at src/gmres.c:281-293), rotates s and decides
// whether the cycle ends.  The host reads back only the small GmresStatus
// record (pinned) after each step, to know whether to queue another one; the
// triangular solve and the x update of src/gmres.c:364-373 are kernels too.
// Every product and sum of the rotations is rounded separately (no fused
// multiply-add), as the reference's BLAS calls compute them.
// ---------------------------------------------------------------------------
struct GmresStatus {
  double resid;   // |s_i| / ||b|| after the last step, or the restart residual
  double rnorm;   // norm of the preconditioned residual at the cycle start
  int i;          // columns of the current cycle
  int iters;      // Arnoldi steps so far
  int state;      // 0 running, 1 converged, 2 cycle full (i == restart or iters == maxit), 3 zero/NaN residual
  int pad;
};

__device__ __forceinline__ void drot_d(double *x, double *y, double cc, double ss) {
  const double xv = *x, yv = *y;
  *x = __dadd_rn(__dmul_rn(cc, xv), __dmul_rn(ss, yv));
  *y = __dsub_rn(__dmul_rn(cc, yv), __dmul_rn(ss, xv));
}

__device__ void drotg_d(double *a, double *b, double *cc, double *ss) {
  const double aa = *a, bb = *b;
  const double roe = (fabs(aa) > fabs(bb)) ? aa : bb;
  const double scale = __dadd_rn(fabs(aa), fabs(bb));
  double r, z;
  if (scale == 0.0) {
    *cc = 1.0; *ss = 0.0; r = 0.0; z = 0.0;
  } else {
    const double ua = __ddiv_rn(aa, scale), ub = __ddiv_rn(bb, scale);
    r = __dmul_rn(scale, __dsqrt_rn(__dadd_rn(__dmul_rn(ua, ua), __dmul_rn(ub, ub))));
    if (roe < 0.0) r = -r;
    *cc = __ddiv_rn(aa, r);
    *ss = __ddiv_rn(bb, r);
    z = 1.0;
    if (fabs(aa) > fabs(bb)) z = *ss;
    if (fabs(bb) >= fabs(aa) && *cc != 0.0) z = __ddiv_rn(1.0, *cc);
  }
  *a = r;
  *b = z;
}

// Cycle start: rnorm = sqrt(sum of the dot partials of r.r); the restart
// residual test of src/gmres.c:225-232 / :352-356 (strict < tol at the very
// first test, <= at a restart); s = (rnorm, 0, ...).
__global__ void gmres_cycle_start_kernel(const double *__restrict__ part, int nPart, double bnrm2, double tol,
                                         int first, int restrt, double *sv, GmresStatus *st) {
  __shared__ double red[kRedThreads];
  double s = 0.0;
  for (int k = threadIdx.x; k < nPart; k += blockDim.x) s += part[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int m = blockDim.x / 2; m > 0; m >>= 1) {
    if ((int)threadIdx.x < m) red[threadIdx.x] += red[threadIdx.x + m];
    __syncthreads();
  }
  const double rn = sqrt(red[0]);
  for (int k = threadIdx.x; k < restrt + 2; k += blockDim.x) sv[k] = (k == 0) ? rn : 0.0;
  if (threadIdx.x == 0) {
    const double res = rn / bnrm2;
    st->rnorm = rn;
    st->resid = res;
    st->i = 0;
    if (first ? (res < tol) : (res <= tol)) st->state = 1;
    else if (!(rn > 0.0) || rn != rn) st->state = 3;
    else st->state = 0;
  }
}

// One Givens step for column i (1-based, as src/gmres.c): H(:, i-1) = h,
// previous rotations, the new rotation, s rotated, residual estimate.  A step
// queued after the cycle ended (state != 0) changes nothing.
__global__ void gmres_givens_kernel(const double *__restrict__ h, double *H, int ldh, int restrt, double *sv,
                                    int i, int iters, int maxit, double bnrm2, double tol, GmresStatus *st) {
  if (threadIdx.x != 0 || st->state != 0) return;
  double *cs = H + (size_t)restrt * ldh, *sn = H + (size_t)(restrt + 1) * ldh;
  double *hc = H + (size_t)(i - 1) * ldh;
  for (int k = 0; k <= i; k++) hc[k] = h[k];
  for (int k = 0; k < i - 1; k++) drot_d(&hc[k], &hc[k + 1], cs[k], sn[k]);
  double aa = hc[i - 1], bb = hc[i];
  drotg_d(&aa, &bb, &cs[i - 1], &sn[i - 1]);
  drot_d(&hc[i - 1], &hc[i], cs[i - 1], sn[i - 1]);
  drot_d(&sv[i - 1], &sv[i], cs[i - 1], sn[i - 1]);
  const double res = fabs(sv[i]) / bnrm2;
  st->resid = res;
  st->i = i;
  st->iters = iters;
  if (res <= tol) st->state = 1;
  else if (iters == maxit || i >= restrt) st->state = 2;
}

// y = H(0:k, 0:k)^-1 s (upper triangular, netlib dtrsv order), k = st->i
__global__ void gmres_trsv_kernel(const double *__restrict__ H, int ldh, const double *__restrict__ sv, double *y,
                                  const GmresStatus *st) {
  if (threadIdx.x != 0) return;
  const int k = st->i;
  for (int j = 0; j < k; j++) y[j] = sv[j];
  for (int j = k - 1; j >= 0; j--) {
    if (y[j] != 0.0) {
      y[j] = __ddiv_rn(y[j], H[(size_t)j * ldh + j]);
      const double t = y[j];
      for (int r = j - 1; r >= 0; r--) y[r] = __dsub_rn(y[r], __dmul_rn(t, H[(size_t)j * ldh + r]));
    }
  }
}

// x += V y over the first st->i columns
__global__ void gmres_update_kernel(long long n, const double *__restrict__ V, long long ldv,
                                    const double *__restrict__ y, const GmresStatus *st, double *x) {
  const int k = st->i;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = x[i];
    for (int j = 0; j < k; j++) s += y[j] * V[(size_t)j * ldv + i];
    x[i] = s;
  }
}

static bool gmres_log_enabled() {
  static const bool on = [] {
    const char *e = getenv("FABIPB_GMRES_LOG_RESID");
    return e != nullptr && atoi(e) > 0;
  }();
  return on;
}

// the status record to the host (pinned), after everything queued so far.
// The host spins on an event query rather than blocking in a stream
// synchronize: a thread put to sleep by a blocking wait can take milliseconds
// to be woken, once per Arnoldi step (measured: GMRES at 204,800 panels 10.7 to
// 57 ms from run to run when blocking, 10.7 to 12.9 when the host stays busy).
static bool read_status(Context &c, const GmresStatus *d_st, GmresStatus *h_st) {
  PrecondDev &p = *c.pc;
  if (!p.evStatus) FB_CUDA(cudaEventCreateWithFlags(&p.evStatus, cudaEventDisableTiming));
  FB_CUDA(cudaMemcpyAsync(h_st, d_st, sizeof(GmresStatus), cudaMemcpyDeviceToHost, c.stream));
  FB_CUDA(cudaEventRecord(p.evStatus, c.stream));
  cudaError_t e;
  while ((e = cudaEventQuery(p.evStatus)) == cudaErrorNotReady) {
  }
  FB_CUDA(e);
  return true;
}

// x := x + V y with y from the device triangular solve
static bool gmres_update_dev(Context &c, int ldh, const GmresStatus *d_st, double *x) {
  PrecondDev &p = *c.pc;
  const long long n2 = 2LL * c.n;
  gmres_trsv_kernel<<<1, 32, 0, c.stream>>>(p.d_H, ldh, p.d_sv, p.d_y, d_st);
  gmres_update_kernel<<<kRedBlocks * 4, 256, 0, c.stream>>>(n2, p.d_V, n2, p.d_y, d_st, x);
  c.launches += 2;
  FB_CUDA(cudaGetLastError());
  return true;
}

// Restarted, left-preconditioned GMRES of src/gmres.c:153-362 with every
// vector and the Hessenberg/Givens state on the device.  Residual measure:
// ||P^-1 (b - A x)|| / ||b||, estimated by |s_i| / ||b|| inside a cycle.
bool gmres_solve(Context &c, const double *b, double *x, int restrt, int maxit, double tol, int *iters, double *resid,
                 int *info, bool adjoint, int *steps) {
  FB_CHECK(c.pc != nullptr, "call fabipb_b200_precond_setup before solving (mode -1 for none)");
  FB_CHECK(restrt >= 1, "GMRES restart must be at least 1");
  PrecondDev &p = *c.pc;
  const long long n2 = 2LL * c.n;
  const int ldh = restrt + 1;
  cudaStream_t s = c.stream;
  if (p.restart != restrt || p.d_V == nullptr) {
    p.restart = restrt;
    if (!p.arena.alloc_n(&p.d_V, (size_t)n2 * (restrt + 1)) || !p.arena.alloc_n(&p.d_r, (size_t)n2) ||
        !p.arena.alloc_n(&p.d_av, (size_t)n2) || !p.arena.alloc_n(&p.d_w, (size_t)n2) ||
        !p.arena.alloc_n(&p.d_h, (size_t)ldh + 1) || !p.arena.alloc_n(&p.d_part, 2 * (size_t)kRedBlocks + 2) ||
        !p.arena.alloc_n(&p.d_y, (size_t)restrt + 1) || !p.arena.alloc_n(&p.d_H, (size_t)ldh * (restrt + 2)) ||
        !p.arena.alloc_n(&p.d_sv, (size_t)restrt + 2) || !p.arena.alloc(&p.d_status, sizeof(GmresStatus)))
      return false;
    if (!p.h_status) FB_CUDA(cudaMallocHost(&p.h_status, 4 * sizeof(GmresStatus)));
  }
  GmresStatus *d_st = static_cast<GmresStatus *>(p.d_status);
  GmresStatus *h_st = static_cast<GmresStatus *>(p.h_status);
  const bool logResid = gmres_log_enabled();
  *info = 0;
  *iters = maxit;
  *resid = tol;
  // ||x0|| decides whether b - A x0 needs the operator; ||b|| scales the test
  double *norms = static_cast<double *>(p.h_status) + 2 * sizeof(GmresStatus) / sizeof(double);
  if (!dot_dev(c, n2, x, x, p.d_part + kRedBlocks, true)) return false;
  if (!dot_dev(c, n2, b, b, p.d_part + kRedBlocks + 1, true)) return false;
  FB_CUDA(cudaMemcpyAsync(norms, p.d_part + kRedBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaStreamSynchronize(s));   // once per solve
  const double xn = norms[0];
  double bnrm2 = norms[1];
  if (bnrm2 == 0.0) bnrm2 = 1.0;
  FB_CUDA(cudaMemcpyAsync(p.d_av, b, n2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (xn != 0.0) {
    if (!op_matvec(c, -1.0, x, 1.0, p.d_av, adjoint)) return false;
  }
  if (!precond_apply(c, p.d_av, p.d_r, adjoint)) return false;
  int it = 0;
  bool first = true;
  int stepsLocal = 0;
  if (!steps) steps = &stepsLocal;
  *steps = 0;
  for (;;) {
    // cycle start: rnorm, the restart residual test, v_0 = r / rnorm
    dot_partial_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(n2, p.d_r, p.d_r, p.d_part);
    gmres_cycle_start_kernel<<<1, kRedThreads, 0, s>>>(p.d_part, kRedBlocks, bnrm2, tol, first ? 1 : 0, restrt,
                                                       p.d_sv, d_st);
    c.launches += 2;
    FB_CUDA(cudaGetLastError());
    if (!read_status(c, d_st, h_st)) return false;
    if (first && h_st->state == 1) return true;   // converged at x0: iters and resid keep their entry values
    *resid = h_st->resid;
    if (!first && logResid) printf("GMRES residual: iter=%d resid=%e\n", it, h_st->resid);
    if (h_st->state == 1) {
      *iters = it;
      return true;
    }
    if (first) {
      *iters = 0;
      first = false;
    } else if (it == maxit) {
      *iters = it;
      *info = 1;
      return true;
    }
    if (h_st->state == 3) {
      const double rn = h_st->rnorm;
      *resid = (rn != rn) ? rn : 0.0;
      *info = (rn != rn) ? 2 : 0;
      *iters = it;
      return true;
    }
    scale_copy_dev_kernel<<<kRedBlocks * 4, 256, 0, s>>>(n2, &d_st->rnorm, p.d_r, p.d_V);
    c.launches += 1;
    int i = 0;
    for (;;) {
      ++i;
      ++it;
      *steps = it;
      if (!op_matvec(c, 1.0, p.d_V + (size_t)(i - 1) * n2, 0.0, p.d_av, adjoint)) return false;
      if (!precond_apply(c, p.d_av, p.d_w, adjoint)) return false;
      // modified Gram-Schmidt: h[k] = w.v_k; w -= h[k] v_k, one launch per
      // column with the partial sums ping-ponged between two buffers
      double *partA = p.d_part, *partB = p.d_part + kRedBlocks;
      dot_partial_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(n2, p.d_w, p.d_V, partA);
      for (int k = 0; k < i; k++) {
        const double *vnext = (k + 1 < i) ? p.d_V + (size_t)(k + 1) * n2 : nullptr;
        mgs_step_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(n2, partA, p.d_h + k, p.d_V + (size_t)k * n2, vnext,
                                                           p.d_w, partB);
        std::swap(partA, partB);
      }
      mgs_norm_scale_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(n2, partA, p.d_h + i, p.d_w,
                                                               p.d_V + (size_t)i * n2);
      gmres_givens_kernel<<<1, 32, 0, s>>>(p.d_h, p.d_H, ldh, restrt, p.d_sv, i, it, maxit, bnrm2, tol, d_st);
      c.launches += i + 3;
      FB_CUDA(cudaGetLastError());
      if (!read_status(c, d_st, h_st)) return false;
      *resid = h_st->resid;
      if (logResid) printf("GMRES residual: iter=%d resid=%e\n", it, h_st->resid);
      if (h_st->state == 1) {
        *iters = it;
        return gmres_update_dev(c, ldh, d_st, x);
      }
      if (h_st->state != 0) break;
    }
    // end of a cycle: x += V y, r = P^-1 (b - A x)
    if (!gmres_update_dev(c, ldh, d_st, x)) return false;
    FB_CUDA(cudaMemcpyAsync(p.d_av, b, n2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (!op_matvec(c, -1.0, x, 1.0, p.d_av, adjoint)) return false;
    if (!precond_apply(c, p.d_av, p.d_r, adjoint)) return false;
    *iters = it;
  }
}

}  // namespace fb

namespace fb {

__global__ void add_kernel(long long n, const double *__restrict__ d, double *x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] += d[i];
}

// Mixed-precision iterative refinement.  First the whole system A x = b is
// solved from the given x by GMRES with the context's own operator (the FP32
// P2P in a mixed context), to tolInner, or to 0.9 of the outer tolerance when
// tolInner is not looser than tol (the FP32 operator's error then rarely lifts
// the FP64 residual above tol); then, until ||P^-1 r|| / ||b|| <= tol (the
// reference GMRES measure, src/gmres.c:225-232), the residual r = b - A x is
// formed with the FP64 operator (in a mixed context the FP64 near-field P2P),
// the correction A d = r is solved by GMRES with the context's operator from
// d = 0, and x += d.  The outer residuals and updates are FP64 vectors.  A
// correction is solved to the relative tolerance tolInner, or only to half
// the reduction the outer test still needs when that is looser: the inner
// GMRES stops at ||P^-1 r_inner|| <= tolStep ||r||, so tolStep =
// 0.5 tol ||b|| / ||r|| leaves the next outer residual near tol / 2, and a
// residual just above tol costs a few inner iterations, not a full tolInner
// reduction far below tol.  When the first solve already meets tol in FP64
// terms, the whole refined solve costs one FP64 residual more than the plain
// solve.
bool refined_solve(Context &c, const double *b, double *x, int restart, int maxit, double tolInner, double tol,
                   int maxOuter, int *outer, int *iters, double *resid, int *info) {
  FB_CHECK(c.pc != nullptr, "call fabipb_b200_precond_setup before solving (mode -1 for none)");
  const long long n2 = 2LL * c.n;
  if (!c.d_refR && (!c.arena.alloc_n(&c.d_refR, (size_t)n2) || !c.arena.alloc_n(&c.d_refD, (size_t)n2) ||
                    !c.arena.alloc_n(&c.d_refZ, (size_t)n2)))
    return false;
  double bn = 0.0;
  if (!dot_to_host(c, n2, b, b, &bn)) return false;
  bn = sqrt(bn);
  if (bn == 0.0) bn = 1.0;
  *outer = 0;
  *iters = 0;
  *info = 0;
  {   // the first solve: the full system from x, on the context's operator
    int it = 0, inf = 0, st = 0;
    double res = 0.0;
    const double tolFirst = tolInner > tol ? tolInner : 0.9 * tol;
    if (!gmres_solve(c, b, x, restart, maxit, tolFirst, &it, &res, &inf, false, &st)) return false;
    *iters += st;
    ++(*outer);
  }
  for (;;) {
    FB_CUDA(cudaMemcpyAsync(c.d_refR, b, n2 * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    if (!op_matvec(c, -1.0, x, 1.0, c.d_refR, false, true)) return false;
    if (!precond_apply(c, c.d_refR, c.d_refZ)) return false;
    double zn = 0.0;
    if (!dot_to_host(c, n2, c.d_refZ, c.d_refZ, &zn)) return false;
    *resid = sqrt(zn) / bn;
    if (*resid <= tol || !(*resid == *resid)) {
      if (!(*resid == *resid)) *info = 2;
      return true;
    }
    if (*outer >= maxOuter || *iters >= maxit) {
      *info = 1;
      return true;
    }
    ++(*outer);
    FB_CUDA(cudaMemsetAsync(c.d_refD, 0, n2 * sizeof(double), c.stream));
    int it = 0, inf = 0;
    double res = 0.0;
    double rn = 0.0;
    if (!dot_to_host(c, n2, c.d_refR, c.d_refR, &rn)) return false;
    rn = sqrt(rn);
    const double tolStep = rn > 0.0 ? fmax(tolInner, 0.5 * tol * bn / rn) : tolInner;
    int st = 0;
    if (!gmres_solve(c, c.d_refR, c.d_refD, restart, maxit - *iters, tolStep, &it, &res, &inf, false, &st))
      return false;
    *iters += st;
    add_kernel<<<kRedBlocks * 4, 256, 0, c.stream>>>(n2, c.d_refD, x);
    c.launches += 1;
    FB_CUDA(cudaGetLastError());
  }
}

}  // namespace fb
