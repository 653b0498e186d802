// adjoint.cu -- gradients of the solvation energy with respect to the
// charges (values and positions), the surface held fixed.
//
// With the direct (exact) panel-charge sums, the discrete energy is
//   E = e(q, r) . sigma,   (D - K) sigma = b(q, r),
// where b is the direct right-hand side (src/fabipb.c:744, the panelRHS
// kernel of src/numQuad.c:786) and e the direct energy weights
// (src/treecode.c:581-661 with every cluster opened):
//   e_pot[X]  = 2 A_X sum_w t w w sum_k q_k (eps dGk/dn - dG0/dn)(x_w - r_k)
//   e_dpdn[X] = 2 A_X sum_w t w w sum_k q_k (G0 - Gk)(x_w - r_k).
// Both are linear in q, so with the adjoint solution (D - K)^T lambda = e
//   dE/dq_k = phi_k = sum_X,w [ e-kernel(x_w - r_k) . sigma + b-kernel(x_w - r_k) . lambda ],
//   dE/dr_k = q_k grad_{r_k} phi_k,
// evaluated by direct sums over the surface quadrature points.  The adjoint
// solve builds its own Krylov basis (nothing of the forward solve is kept but
// sigma).  There is no counterpart in the reference, which has no gradients.

namespace fb {

// Direct energy weights (pot slot: eps dGk/dn - dG0/dn, dpdn slot: G0 - Gk),
// with the tiling of rhs_direct_kernel.
__global__ void energy_weights_kernel(int n, int m, int q, const double *__restrict__ vtx,
                                      const double *__restrict__ nrm, const double *__restrict__ area,
                                      const double *__restrict__ pos, const double *__restrict__ chr, double kappa,
                                      double eps, double *out) {
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
      sc[j] = make_double4(pos[3 * (size_t)(base + j)], pos[3 * (size_t)(base + j) + 1],
                           pos[3 * (size_t)(base + j) + 2], chr[base + j]);
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
          const double ip = nx[0] * r[0] + nx[1] * r[1] + nx[2] * r[2];
          const double tw = t[ix] * w[ix] * w[jx];
          const double rn = sqrt(r2), G0 = kFourPiI / rn, ek = exp(-kappa * rn);
          const double dG0dn = -ip * G0 / r2;
          i0 += (G0 - ek * G0) * tw;                                   // G0 - Gk
          i1 += (eps * (kappa * rn + 1.0) * ek - 1.0) * dG0dn * tw;    // eps dGk/dn - dG0/dn
        }
      s0 += cj.w * (i0 * A2);
      s1 += cj.w * (i1 * A2);
    }
    __syncthreads();
  }
  if (!valid) return;
  out[X] = s1;       // pot slot
  out[n + X] = s0;   // dpdn slot
}

// Mixed contexts, one-point rule: the same weights with FP32 pair terms
// (positions relative to the root box centre, MUFU rsqrt/exp2) in packed
// f32x2 arithmetic, two charges per step (charge pairs staged as
// rhs_direct_f2_kernel stages them), summed in FP32 over 64 charges at a time
// and in FP64 above.  The pair sums leave out the common factor 1/(4 pi)
// (and the sign of dG0/dn), which the FP64 epilogue applies:
//   dpdn: sum q (1 - e)/r,   pot: -sum q (eps (kappa r + 1) e - 1) (n.d)/r^3.
__global__ void __launch_bounds__(256)
energy_weights_f2_kernel(int n, int m, const double *__restrict__ vtx, const double *__restrict__ nrm,
                         const double *__restrict__ area, const float4 *__restrict__ chg, double ox, double oy,
                         double oz, float kappa, float kexp, float eps, double *out) {
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
  const float2 ek = f2(eps * kappa), ev = f2(eps), m1 = f2(-1.f), ke = f2(kexp);
  double s0 = 0.0, s1 = 0.0;
  for (int base = 0; base < m; base += kRhsTileF) {
    const int cnt = min(kRhsTileF, m - base), cnt2 = (cnt + 1) / 2;
    stage_charge_pairs(chg, base, cnt, sc);
    __syncthreads();
    for (int j0 = 0; j0 < cnt2; j0 += 32) {
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
        const float2 r = __fmul2_rn(r2, ri);
        const float2 ea = __fmul2_rn(ke, r);
        float2 e;
        e.x = expneg_t(1.f, ea.x);
        e.y = expneg_t(1.f, ea.y);
        a0 = __ffma2_rn(q, __ffma2_rn(make_float2(-e.x, -e.y), ri, ri), a0);   // q (G0 - Gk) 4 pi
        const float2 ip = __ffma2_rn(nz, dz, __ffma2_rn(ny, dy, __fmul2_rn(nx, dx)));
        const float2 w = __fmul2_rn(ip, __fmul2_rn(__fmul2_rn(ri, ri), ri));
        const float2 u = __ffma2_rn(__ffma2_rn(ek, r, ev), e, m1);           // eps c - 1
        a1 = __ffma2_rn(q, __fmul2_rn(u, w), a1);
      }
      s0 += (double)a0.x + (double)a0.y;
      s1 += (double)a1.x + (double)a1.y;
    }
    __syncthreads();
  }
  if (!valid) return;
  const double W = 2.0 * area[Xs] * t * wt * wt * kFourPiI;
  out[X] = -s1 * W;     // pot slot
  out[n + X] = s0 * W;  // dpdn slot
}

// Per surface quadrature point: position, normal and the four weights
//   a1 = 2A t w w sigma_dpdn, a2 = 2A t w w sigma_pot,
//   a3 = 2A t w w fac lambda_pot, a4 = 2A t w w fac lambda_dpdn.
__global__ void grad_records_kernel(int n, int q, const double *__restrict__ vtx, const double *__restrict__ nrm,
                                    const double *__restrict__ area, const double *__restrict__ sgm,
                                    const double *__restrict__ lam, double fac, double4 *rp, double4 *rn, double2 *rw) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const int qq = q * q;
  if (id >= n * qq) return;
  const int X = id / qq, ix = (id % qq) / q, jx = id % q;
  const double *v0 = vtx + 9 * (size_t)X;
  const double *t = c_tLeg[q], *w = c_wLeg[q];
  double p[3];
  for (int k = 0; k < 3; k++) {
    const double ax2 = v0[3 + k] - v0[k], ax0 = v0[6 + k] - v0[3 + k];
    p[k] = v0[k] + t[ix] * (ax2 + t[jx] * ax0);
  }
  const double a = 2.0 * area[X] * t[ix] * w[ix] * w[jx];
  rp[id] = make_double4(p[0], p[1], p[2], a * sgm[n + X]);
  rn[id] = make_double4(nrm[3 * (size_t)X], nrm[3 * (size_t)X + 1], nrm[3 * (size_t)X + 2], a * sgm[X]);
  rw[id] = make_double2(a * fac * lam[X], a * fac * lam[n + X]);
}

// The records of a mixed context, one-point rule, in FP32, with the weights
// pre-combined for charge_grad_f2_kernel (f = 1/(4 pi), a_i as above) and two
// records interleaved per 96-byte pair, so that every packed f32x2 operand of
// the pair loop is one half of a float4 of the pair:
//   q[0] = (x0 x1 y0 y1)   position x_w - o
//   q[1] = (z0 z1 a0 a1)   a  = -f a1
//   q[2] = (nx0 nx1 ny0 ny1)
//   q[3] = (nz0 nz1 b0 b1) b  = f a2 eps
//   q[4] = (u0 u1 v0 v1)   u  = f a1 + a3,  v = a4 - f a2
//   q[5] = (s0 s1 w0 w1)   s  = f a1 kappa, w = f a2 eps kappa^2.
// An odd record count pads the last pair with a copy of the last position
// and zero weights and normal, which adds exactly zero.
__global__ void grad_records_f2_kernel(int n, const double *__restrict__ vtx, const double *__restrict__ nrm,
                                       const double *__restrict__ area, const double *__restrict__ sgm,
                                       const double *__restrict__ lam, double fac, double ox, double oy, double oz,
                                       double kappa, double eps, float4 *rq) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (n + 1) / 2) return;
  const double t = c_tLeg[1][0], w = c_wLeg[1][0];
  float v[2][12];
  for (int h = 0; h < 2; h++) {
    const int X = min(2 * j + h, n - 1);
    const double live = 2 * j + h < n ? 1.0 : 0.0;
    const double *v0 = vtx + 9 * (size_t)X;
    double p[3];
    for (int k = 0; k < 3; k++) p[k] = v0[k] + t * ((v0[3 + k] - v0[k]) + t * (v0[6 + k] - v0[3 + k]));
    const double a = live * 2.0 * area[X] * t * w * w;
    const double f1 = kFourPiI * a * sgm[n + X], f2v = kFourPiI * a * sgm[X];
    const double a3 = a * fac * lam[X], a4 = a * fac * lam[n + X];
    float *o = v[h];
    o[0] = (float)(p[0] - ox);
    o[1] = (float)(p[1] - oy);
    o[2] = (float)(p[2] - oz);
    o[3] = (float)(-f1);
    for (int k = 0; k < 3; k++) o[4 + k] = (float)(live * nrm[3 * (size_t)X + k]);
    o[7] = (float)(f2v * eps);
    o[8] = (float)(f1 + a3);
    o[9] = (float)(a4 - f2v);
    o[10] = (float)(f1 * kappa);
    o[11] = (float)(f2v * eps * kappa * kappa);
  }
  float4 *q = rq + 6 * (size_t)j;
  for (int s = 0; s < 6; s++) q[s] = make_float4(v[0][2 * s], v[1][2 * s], v[0][2 * s + 1], v[1][2 * s + 1]);
}

constexpr int kGradCharges = 128;   // threads per block (FP64 kernel: charges per block)
constexpr int kGradTile = 128;      // records staged per step
constexpr int kGradCpt = 2;         // charges per thread in charge_grad_f2_kernel

// One record pair against one charge (c = the negated charge position), in
// packed f32x2 arithmetic.  With A = f a1 (1 - e) + a3 and B = f a2 (eps c - 1)
// + a4 (e = exp(-kappa r), c = (kappa r + 1) e), the record's term and its
// gradient in x = x_w - r_k are
//   phi  = A/r - (n.x) B/r^3,
//   grad = x [f a1 kappa e/r^2 - A/r^3 + (n.x)/r^3 (3B/r^2 + f a2 eps kappa^2 e)] - n B/r^3.
__device__ __forceinline__ void grad_pair2(const float4 Q0, const float4 Q1, const float4 Q2, const float4 Q3,
                                           const float4 Q4, const float4 Q5, float2 cx, float2 cy, float2 cz,
                                           float kappa, float kexp, float2 &phi, float2 &gx, float2 &gy,
                                           float2 &gz) {
  const float2 x = __fadd2_rn(make_float2(Q0.x, Q0.y), cx);
  const float2 y = __fadd2_rn(make_float2(Q0.z, Q0.w), cy);
  const float2 z = __fadd2_rn(make_float2(Q1.x, Q1.y), cz);
  const float2 r2 = __ffma2_rn(z, z, __ffma2_rn(y, y, __fmul2_rn(x, x)));
  float2 ri;
  ri.x = rsqrt_t(r2.x);
  ri.y = rsqrt_t(r2.y);
  const float2 r = __fmul2_rn(r2, ri), ri2 = __fmul2_rn(ri, ri), ri3 = __fmul2_rn(ri2, ri);
  const float2 ea = __fmul2_rn(f2(kexp), r);
  float2 e;
  e.x = expneg_t(1.f, ea.x);
  e.y = expneg_t(1.f, ea.y);
  const float2 c = __fmul2_rn(__ffma2_rn(f2(kappa), r, f2(1.f)), e);
  const float2 nx = make_float2(Q2.x, Q2.y), ny = make_float2(Q2.z, Q2.w), nz = make_float2(Q3.x, Q3.y);
  const float2 ip = __ffma2_rn(nz, z, __ffma2_rn(ny, y, __fmul2_rn(nx, x)));
  const float2 A = __ffma2_rn(make_float2(Q1.z, Q1.w), e, make_float2(Q4.x, Q4.y));
  const float2 B = __ffma2_rn(make_float2(Q3.z, Q3.w), c, make_float2(Q4.z, Q4.w));
  const float2 t = __fmul2_rn(ip, ri3);
  phi = __ffma2_rn(A, ri, phi);
  phi = __ffma2_rn(make_float2(-t.x, -t.y), B, phi);
  const float2 u = __ffma2_rn(__fmul2_rn(f2(3.f), ri2), B, __fmul2_rn(make_float2(Q5.z, Q5.w), e));
  const float2 sxv = __ffma2_rn(__fmul2_rn(make_float2(Q5.x, Q5.y), e), ri2,
                                __ffma2_rn(make_float2(-A.x, -A.y), ri3, __fmul2_rn(t, u)));
  const float2 snv = __fmul2_rn(make_float2(-ri3.x, -ri3.y), B);
  gx = __ffma2_rn(sxv, x, __ffma2_rn(snv, nx, gx));
  gy = __ffma2_rn(sxv, y, __ffma2_rn(snv, ny, gy));
  gz = __ffma2_rn(sxv, z, __ffma2_rn(snv, nz, gz));
}

// charge_grad_kernel with FP32 pair terms (records and charges relative to
// the root box centre) in packed f32x2 arithmetic: every thread takes two
// charges (k and k + 128) and every step one record pair, so each staged
// float4 feeds four pair terms.  FP32 sums over 64 records at a time, FP64
// above; part[chunk][k] as charge_grad_kernel.
__global__ void __launch_bounds__(kGradCharges)
charge_grad_f2_kernel(long long nPairs, int m, long long chunkPairs, const float4 *__restrict__ rq,
                      const float4 *__restrict__ chg, float kappa, float kexp, double4 *part) {
  constexpr int kPairs = kGradTile / 2;
  __shared__ float4 sq[6 * kPairs];
  float2 cx[kGradCpt], cy[kGradCpt], cz[kGradCpt];
  double phi[kGradCpt], gx[kGradCpt], gy[kGradCpt], gz[kGradCpt];
#pragma unroll
  for (int h = 0; h < kGradCpt; h++) {
    const int k = blockIdx.x * (kGradCharges * kGradCpt) + h * kGradCharges + threadIdx.x;
    const float4 ck = k < m ? chg[k] : make_float4(0.f, 0.f, 0.f, 0.f);
    cx[h] = f2(-ck.x);
    cy[h] = f2(-ck.y);
    cz[h] = f2(-ck.z);
    phi[h] = gx[h] = gy[h] = gz[h] = 0.0;
  }
  const long long p0 = (long long)blockIdx.y * chunkPairs, p1 = min(nPairs, p0 + chunkPairs);
  for (long long b = p0; b < p1; b += kPairs) {
    const int cnt = (int)min((long long)kPairs, p1 - b);
    for (int i = threadIdx.x; i < 6 * cnt; i += blockDim.x) sq[i] = rq[6 * b + i];
    __syncthreads();
    for (int j0 = 0; j0 < cnt; j0 += 32) {
      const int j1 = min(cnt, j0 + 32);
      float2 fphi[kGradCpt], fx[kGradCpt], fy[kGradCpt], fz[kGradCpt];
#pragma unroll
      for (int h = 0; h < kGradCpt; h++) fphi[h] = fx[h] = fy[h] = fz[h] = f2(0.f);
#pragma unroll 2
      for (int j = j0; j < j1; j++) {
        const float4 Q0 = sq[6 * j], Q1 = sq[6 * j + 1], Q2 = sq[6 * j + 2], Q3 = sq[6 * j + 3],
                     Q4 = sq[6 * j + 4], Q5 = sq[6 * j + 5];
#pragma unroll
        for (int h = 0; h < kGradCpt; h++)
          grad_pair2(Q0, Q1, Q2, Q3, Q4, Q5, cx[h], cy[h], cz[h], kappa, kexp, fphi[h], fx[h], fy[h], fz[h]);
      }
#pragma unroll
      for (int h = 0; h < kGradCpt; h++) {
        phi[h] += (double)fphi[h].x + (double)fphi[h].y;
        gx[h] += (double)fx[h].x + (double)fx[h].y;
        gy[h] += (double)fy[h].x + (double)fy[h].y;
        gz[h] += (double)fz[h].x + (double)fz[h].y;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int h = 0; h < kGradCpt; h++) {
    const int k = blockIdx.x * (kGradCharges * kGradCpt) + h * kGradCharges + threadIdx.x;
    if (k < m) part[(size_t)blockIdx.y * m + k] = make_double4(phi[h], -gx[h], -gy[h], -gz[h]);   // d/dr_k = -d/dx
  }
}

// phi_k and grad_{r_k} phi_k over one chunk of the records, for a tile of
// charges (one thread per charge); part[chunk][k] = (phi, grad).
__global__ void __launch_bounds__(kGradCharges)
charge_grad_kernel(long long nRec, int m, long long chunkLen, const double4 *__restrict__ rp,
                   const double4 *__restrict__ rn, const double2 *__restrict__ rw, const double *__restrict__ pos,
                   double kappa, double eps, double4 *part) {
  __shared__ double4 sp[kGradTile], sn[kGradTile];
  __shared__ double2 sw[kGradTile];
  const int k = blockIdx.x * kGradCharges + threadIdx.x;
  const bool valid = k < m;
  const double px = valid ? pos[3 * (size_t)k] : 0.0, py = valid ? pos[3 * (size_t)k + 1] : 0.0,
               pz = valid ? pos[3 * (size_t)k + 2] : 0.0;
  const long long r0 = (long long)blockIdx.y * chunkLen, r1 = min(nRec, r0 + chunkLen);
  const double kap2 = kappa * kappa;
  double phi = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;   // gradient with respect to x = x_w - r_k
  for (long long b = r0; b < r1; b += kGradTile) {
    const int cnt = (int)min((long long)kGradTile, r1 - b);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      sp[j] = rp[b + j];
      sn[j] = rn[b + j];
      sw[j] = rw[b + j];
    }
    __syncthreads();
    for (int j = 0; j < cnt; j++) {
      const double4 P = sp[j], N = sn[j];
      const double2 W = sw[j];
      const double x = P.x - px, y = P.y - py, z = P.z - pz;
      const double r2 = x * x + y * y + z * z;
      const double ri = 1.0 / sqrt(r2), r = r2 * ri, ri2 = ri * ri, ri3 = ri2 * ri;
      const double ip = N.x * x + N.y * y + N.z * z;
      const double G0 = kFourPiI * ri;
      const double e = exp(-kappa * r), c = (kappa * r + 1.0) * e;
      const double dG0dn = -kFourPiI * ip * ri3;
      // a1 (G0 - Gk) + a2 (eps c - 1) dG0/dn + a3 / r - a4 ip / r^3
      phi += P.w * (G0 - e * G0) + N.w * (eps * c - 1.0) * dG0dn + W.x * ri - W.y * ip * ri3;
      // gradients in x
      const double fG = -P.w * (1.0 - c) * G0 * ri2;   // grad (G0 - Gk) = -(1 - c) G0 x / r^2
      const double h5 = 3.0 * ip * ri2 * ri3;           // 3 ip / r^5
      // grad dG0/dn = -(1/4pi) (n/r^3 - 3 ip x/r^5); grad c = -kappa^2 e x
      const double cn = N.w * (eps * c - 1.0) * (-kFourPiI), cx = N.w * (-eps * kap2 * e) * dG0dn;
      const double an = -W.y;                            // grad(-ip/r^3) = -(n/r^3 - 3 ip x/r^5)
      const double sx = fG + cx - cn * h5 - W.x * ri3 - an * h5;
      const double sn_ = cn * ri3 + an * ri3;
      gx += sx * x + sn_ * N.x;
      gy += sx * y + sn_ * N.y;
      gz += sx * z + sn_ * N.z;
    }
    __syncthreads();
  }
  if (valid) part[(size_t)blockIdx.y * m + k] = make_double4(phi, -gx, -gy, -gz);   // d/dr_k = -d/dx
}

__global__ void charge_grad_reduce_kernel(int m, int nChunks, const double4 *__restrict__ part,
                                          const double *__restrict__ chr, double scale, double *dEdq, double *dEdx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double phi = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  for (int c = 0; c < nChunks; c++) {
    const double4 v = part[(size_t)c * m + k];
    phi += v.x;
    gx += v.y;
    gy += v.z;
    gz += v.w;
  }
  if (dEdq) dEdq[k] = scale * phi;
  if (dEdx) {
    const double s = scale * chr[k];
    dEdx[3 * (size_t)k] = s * gx;
    dEdx[3 * (size_t)k + 1] = s * gy;
    dEdx[3 * (size_t)k + 2] = s * gz;
  }
}

struct AdjointDev {
  DevArena arena;
  double *d_b = nullptr, *d_sigma = nullptr, *d_e = nullptr, *d_lam = nullptr, *d_out = nullptr;
  double4 *d_rp = nullptr, *d_rn = nullptr, *d_part = nullptr;
  double2 *d_rw = nullptr;
  float4 *d_rq = nullptr;
  long long recCap = 0, rqCap = 0, partCap = 0;
  int outCap = 0;
  bool forwardDone = false;
  double energy = 0.0;
};

void free_adjoint(Context &c) {
  if (c.adj) {
    c.adj->arena.release();
    delete c.adj;
    c.adj = nullptr;
  }
}

static bool adj_state(Context &c) {
  if (!c.adj) c.adj = new AdjointDev();
  AdjointDev &a = *c.adj;
  if (!a.d_b) {
    const size_t n2 = 2 * (size_t)c.n;
    if (!a.arena.alloc_n(&a.d_b, n2) || !a.arena.alloc_n(&a.d_sigma, n2) || !a.arena.alloc_n(&a.d_e, n2) ||
        !a.arena.alloc_n(&a.d_lam, n2))
      return false;
  }
  return true;
}

bool launch_energy_weights(Context &c, double *e) {
  FB_CHECK(c.ct != nullptr && c.nChar > 0, "no charges set (fabipb_b200_set_charges)");
  FB_CHECK(c.prm.quad_order >= 1 && c.prm.quad_order <= 10, "quadrature order %d outside 1..10", c.prm.quad_order);
  if (c.mixed && c.prm.quad_order == 1) {
    double ox, oy, oz;
    if (!charges_f32(c, &ox, &oy, &oz)) return false;
    energy_weights_f2_kernel<<<ceil_div(c.n, 256), 256, 0, c.stream>>>(
        c.n, c.nChar, c.d_vtx, c.d_nrm, c.d_area, c.ct->d_chgF, ox, oy, oz, (float)c.prm.kappa,
        (float)(-c.prm.kappa * 1.4426950408889634), (float)c.epsilon, e);
    c.launches += 1;
    FB_CUDA(cudaGetLastError());
    return true;
  }
  energy_weights_kernel<<<ceil_div(c.n, 128), 128, 0, c.stream>>>(c.n, c.nChar, c.prm.quad_order, c.d_vtx, c.d_nrm,
                                                                  c.d_area, c.ct->d_posOrig, c.ct->d_chrOrig,
                                                                  c.prm.kappa, c.epsilon, e);
  c.launches += 1;
  FB_CUDA(cudaGetLastError());
  return true;
}

// e . x with the deterministic two-pass reduction, result to the host
static bool dot_host(Context &c, const double *x, const double *y, double *out) {
  return dot_to_host(c, 2LL * c.n, x, y, out);
}

bool adjoint_forward(Context &c, int restart, int maxit, double tol, double *energy, int *iters, double *resid,
                     int *info) {
  FB_CHECK(c.ct != nullptr && c.nChar > 0, "no charges set (fabipb_b200_set_charges)");
  if (!adj_state(c)) return false;
  AdjointDev &a = *c.adj;
  a.forwardDone = false;
  if (!c.pc && !precond_setup(c, 2)) return false;
  if (!launch_rhs(c, 0, a.d_b)) return false;
  FB_CUDA(cudaMemcpyAsync(a.d_sigma, a.d_b, 2 * (size_t)c.n * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
  if (!gmres_solve(c, a.d_b, a.d_sigma, restart, maxit, tol, iters, resid, info)) return false;
  if (!launch_energy_weights(c, a.d_e)) return false;
  if (!dot_host(c, a.d_e, a.d_sigma, &a.energy)) return false;
  *energy = a.energy;
  a.forwardDone = true;
  return true;
}

bool adjoint_backward(Context &c, double scale, int restart, int maxit, double tol, double *dEdq, double *dEdx,
                      int *iters, double *resid, int *info) {
  FB_CHECK(c.adj != nullptr && c.adj->forwardDone, "fabipb_b200_backward needs a preceding fabipb_b200_forward");
  AdjointDev &a = *c.adj;
  // lambda: (D - K)^T lambda = e, from lambda0 = e
  FB_CUDA(cudaMemcpyAsync(a.d_lam, a.d_e, 2 * (size_t)c.n * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
  if (!gmres_solve(c, a.d_e, a.d_lam, restart, maxit, tol, iters, resid, info, true)) return false;
  // records, then per-charge sums over chunks of records
  const int q = c.prm.quad_order, m = c.nChar;
  const long long nRec = (long long)c.n * q * q;
  const double fac = c.rhsFac != 0.0 ? c.rhsFac : kFourPiI / c.prm.eps1;
  const bool f32 = c.mixed && q == 1;   // FP32 pair terms, records interleaved in pairs
  const long long nPairs = (nRec + 1) / 2;
  if (f32) {
    if (a.rqCap < 6 * nPairs) {
      if (!a.arena.alloc_n(&a.d_rq, (size_t)(6 * nPairs))) return false;
      a.rqCap = 6 * nPairs;
    }
  } else if (a.recCap < nRec) {
    if (!a.arena.alloc_n(&a.d_rp, (size_t)nRec) || !a.arena.alloc_n(&a.d_rn, (size_t)nRec) ||
        !a.arena.alloc_n(&a.d_rw, (size_t)nRec))
      return false;
    a.recCap = nRec;
  }
  if (f32) {
    double ox, oy, oz;
    if (!charges_f32(c, &ox, &oy, &oz)) return false;
    grad_records_f2_kernel<<<ceil_div(nPairs, 256), 256, 0, c.stream>>>(
        c.n, c.d_vtx, c.d_nrm, c.d_area, a.d_sigma, a.d_lam, fac, ox, oy, oz, c.prm.kappa, c.epsilon, a.d_rq);
  } else {
    grad_records_kernel<<<ceil_div(nRec, 256), 256, 0, c.stream>>>(c.n, q, c.d_vtx, c.d_nrm, c.d_area, a.d_sigma,
                                                                   a.d_lam, fac, a.d_rp, a.d_rn, a.d_rw);
  }
  // enough blocks to fill the GPU: chunks of the records times tiles of charges
  const int perBlock = f32 ? kGradCharges * kGradCpt : kGradCharges;
  const int tiles = (int)ceil_div(m, perBlock);
  const long long want = (2368LL + tiles - 1) / tiles, most = (nRec + 4095) / 4096;
  const int nChunks = (int)std::max(1LL, std::min(want, most));
  const long long chunkPairs = (nPairs + nChunks - 1) / nChunks, chunkLen = (nRec + nChunks - 1) / nChunks;
  if (a.partCap < (long long)nChunks * m) {
    if (!a.arena.alloc_n(&a.d_part, (size_t)nChunks * m)) return false;
    a.partCap = (long long)nChunks * m;
  }
  dim3 grid(tiles, nChunks);
  if (f32)
    charge_grad_f2_kernel<<<grid, kGradCharges, 0, c.stream>>>(nPairs, m, chunkPairs, a.d_rq, c.ct->d_chgF,
                                                               (float)c.prm.kappa,
                                                               (float)(-c.prm.kappa * 1.4426950408889634), a.d_part);
  else
    charge_grad_kernel<<<grid, kGradCharges, 0, c.stream>>>(nRec, m, chunkLen, a.d_rp, a.d_rn, a.d_rw,
                                                           c.ct->d_posOrig, c.prm.kappa, c.epsilon, a.d_part);
  charge_grad_reduce_kernel<<<ceil_div(m, 256), 256, 0, c.stream>>>(m, nChunks, a.d_part, c.ct->d_chrOrig, scale,
                                                                    dEdq, dEdx);
  c.launches += 3;
  FB_CUDA(cudaGetLastError());
  return true;
}

}  // namespace fb

extern "C" {

int fabipb_b200_energy_weights(void *ctx, double *e, int on_device) {
  if (!valid_ctx(ctx) || e == nullptr) return 0;
  Context *c = (Context *)ctx;
  return with_vectors(c, nullptr, e, false, on_device, [&](const double *, double *y) {
    return launch_energy_weights(*c, y);
  });
}

int fabipb_b200_forward(void *ctx, int restart, int maxit, double tol, double *energy_raw, int *iters, double *resid,
                        int *info) {
  if (!valid_ctx(ctx) || energy_raw == nullptr || restart < 1 || maxit < 1) {
    set_error("fabipb_b200_forward: invalid arguments");
    return 0;
  }
  Context *c = (Context *)ctx;
  cudaSetDevice(c->device);
  int it = 0, inf = 0;
  double res = 0.0;
  const bool ok = adjoint_forward(*c, restart, maxit, tol, energy_raw, &it, &res, &inf);
  if (iters) *iters = it;
  if (resid) *resid = res;
  if (info) *info = inf;
  return ok ? 1 : 0;
}

int fabipb_b200_backward(void *ctx, double grad_energy, int restart, int maxit, double tol, double *dEdq,
                         double *dEdx, int *iters, double *resid, int *info, int on_device) {
  if (!valid_ctx(ctx) || restart < 1 || maxit < 1) {
    set_error("fabipb_b200_backward: invalid arguments");
    return 0;
  }
  Context *c = (Context *)ctx;
  cudaSetDevice(c->device);
  const int m = c->nChar;
  double *dq = dEdq, *dx = dEdx;
  if (!on_device) {
    if (!c->adj && !adj_state(*c)) return 0;
    AdjointDev &a = *c->adj;
    if (a.outCap < m) {
      if (!a.arena.alloc_n(&a.d_out, 4 * (size_t)m)) return 0;
      a.outCap = m;
    }
    dq = dEdq ? a.d_out : nullptr;
    dx = dEdx ? a.d_out + m : nullptr;
  }
  int it = 0, inf = 0;
  double res = 0.0;
  bool ok = adjoint_backward(*c, grad_energy, restart, maxit, tol, dq, dx, &it, &res, &inf);
  if (ok && !on_device) {
    if (dEdq) ok = cudaMemcpyAsync(dEdq, dq, m * sizeof(double), cudaMemcpyDeviceToHost, c->stream) == cudaSuccess;
    if (ok && dEdx)
      ok = cudaMemcpyAsync(dEdx, dx, 3 * (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, c->stream) == cudaSuccess;
    if (!ok) set_error("device-to-host copy failed");
  }
  if (ok && cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("backward failed: %s", cudaGetErrorString(cudaGetLastError()));
    ok = false;
  }
  if (iters) *iters = it;
  if (resid) *resid = res;
  if (info) *info = inf;
  return ok ? 1 : 0;
}

}  // extern "C"
