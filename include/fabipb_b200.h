/*
 * fabipb_b200.h -- plain-pointer C ABI of the B200 FABIPB hot path.
 *
 * One context holds a molecular-surface mesh resident on one GPU: the octree
 * (built exactly as the reference's gkInit, src/gkSetup.c:446-508), the leaf
 * moment matrices, the near-field special-pair table and the FMM expansion
 * storage.  Every operator the reference's GMRES matvec uses is then a few
 * kernel launches on vectors that stay in HBM.
 *
 * Conventions (those of the reference):
 *   - panels are given in mesh-face (input) order: vtx[9*i + 3*k + d] is
 *     coordinate d of vertex k, normal[3*i + d], area[i];
 *   - unknown vectors have length 2N in tree (pnlLst) order: entries [0,N)
 *     are the potential part, [N,2N) the normal-derivative part.  The
 *     permutation is returned by fabipb_b200_panel_order();
 *   - every function returns 1 on success and 0 on failure, with a message
 *     in fabipb_b200_last_error() (src/gpu_backend_cuda.cu:320-326 uses the
 *     same 1/0 convention).  There is no CPU fallback anywhere: a failure is
 *     reported, never silently recomputed on the host;
 *   - `on_device` = 1 means the vector pointers are CUDA device pointers on
 *     the context's device; 0 means host pointers (copied in and out inside
 *     the call, the path the reference's plugin ABI takes).
 */
#ifndef FABIPB_B200_H
#define FABIPB_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* arithmetic of the near field and the FMM passes */
#define FABIPB_B200_FP64 0   /* everything in double */
#define FABIPB_B200_MIXED 1  /* near-field P2P in float, singular pairs and
                                the far field in double */

/* which part of the boundary operator K an apply covers */
#define FABIPB_B200_NEAR 1
#define FABIPB_B200_FAR 2
#define FABIPB_B200_ALL 3

typedef struct fabipb_b200_params {
  int order;          /* -p : >0 fixed Taylor order, <=0 variable (gkSetup.c:42) */
  int order_mom;      /* -pm (default 0) */
  int depth;          /* -t : octree depth */
  int height;         /* -H : coarsest FMM level */
  int quad_order;     /* -q : panel quadrature order (the device path needs 1) */
  double sep_ratio;   /* -S : MAC separation ratio */
  double kappa;       /* -k : Debye-Hueckel screening */
  double eps1, eps2;  /* -eps1 -eps2 */
  double rhs_theta;   /* charge-tree acceptance for the RHS (default 0.8) */
  double energy_theta;/* charge-tree acceptance for the energy (default 0.8) */
  int charge_order;   /* charge-tree Taylor order: >0 flat, 0 follow the FMM */
  int precision;      /* FABIPB_B200_FP64 or FABIPB_B200_MIXED */
  int device;         /* CUDA device ordinal */
} fabipb_b200_params;

typedef struct fabipb_b200_info {
  int panels, leaves, near_pairs, m2l_pairs, cubes, max_order, leaf_order;
  int max_leaf;
  long long near_panel_pairs;  /* panel pairs the near field visits per apply */
  long long special_pairs;     /* of those, pairs with a shared vertex/edge or self */
  double setup_seconds;
  double device_bytes;         /* device memory held by the context */
} fabipb_b200_info;

void fabipb_b200_default_params(fabipb_b200_params *p);

int fabipb_b200_create(const fabipb_b200_params *p, int n_panels, const double *vtx,
                       const double *normal, const double *area, void **ctx);
/* The direct operator of the reference's -r modes (MtVmain's direct branch,
   src/fabipb.c:1250-1265, src/direct_backend.c:172): every panel pair through
   the near-field rules, no FMM.  The context takes every call a
   fabipb_b200_create context takes; its matvec, solves and adjoint use the
   O(N^2) sum (an FP64 direct-summation oracle in FP64 precision). */
int fabipb_b200_create_direct(const fabipb_b200_params *p, int n_panels, const double *vtx,
                              const double *normal, const double *area, void **ctx);
int fabipb_b200_set_charges(void *ctx, int n_charges, const double *pos, const double *q);
void fabipb_b200_destroy(void *ctx);
int fabipb_b200_set_stream(void *ctx, void *cuda_stream);
/* number of CUDA kernels this context has launched so far */
long long fabipb_b200_launch_count(void *ctx);
const char *fabipb_b200_last_error(void);
/* Measured FMA rate of a device's FP32 (fp64 = 0: packed f32x2 FMA chains)
   or FP64 (fp64 = 1) pipe in TFLOP/s, best of five event-timed launches: the
   roofline denominators of the FMA-bound near field.  No counterpart in the
   reference. */
int fabipb_b200_simt_peak(int device, int fp64, double *tflops);

/* tree queries, for parity checks against the reference layouts */
int fabipb_b200_info_get(void *ctx, fabipb_b200_info *out);
int fabipb_b200_panel_order(void *ctx, int *order);      /* tree index -> input index (N) */
int fabipb_b200_leaf_layout(void *ctx, int *start, int *count);
int fabipb_b200_near_pairs(void *ctx, int *src, int *dst);   /* fmm.c:234-268 order */
int fabipb_b200_m2l_pairs(void *ctx, int *src, int *dst);    /* fmm.c:326-373 order */
int fabipb_b200_cube_data(void *ctx, int *level, double *ctr4);

/* pot = beta*pot + alpha*K_part*sgm  (applyFMM, src/fmm.c:710, and its
   near/far halves) */
int fabipb_b200_apply(void *ctx, int part, double alpha, const double *sgm, double beta,
                      double *pot, int on_device);
/* y = alpha*(D - K)x + beta*y  (MtVmain, src/fabipb.c:1237) */
int fabipb_b200_matvec(void *ctx, double alpha, const double *x, double beta, double *y,
                       int on_device);
/* iterative refinement (no counterpart in the reference): FP64 residuals
   r = b - A x (in a mixed context through the FP64 near-field P2P), each
   correction solved by GMRES with the context's operator (the FP32 P2P in a
   mixed context) from zero to the relative tolerance tol_inner, or only to
   half the reduction the outer tolerance still needs (0.5 tol ||b|| / ||r||)
   when that is looser, x += d, until ||P^-1 r|| / ||b|| <= tol.  x holds the initial guess.  *outer =
   corrections made, *iters = inner GMRES iterations in total (at most
   maxit), *info = 0 converged, 1 out of iterations, 2 NaN. */
int fabipb_b200_solve_refined(void *ctx, const double *b, double *x, int restart, int maxit, double tol_inner,
                              double tol, int max_outer, int *outer, int *iters, double *resid, int *info,
                              int on_device);
/* stage report (the counterpart of the reference's -B=1 stage times, no
   counterpart in its ABI): runs the matvec passes reps times with CUDA events
   between them and returns the mean milliseconds per pass in ms[6]:
   near field (pack + P2P + FP64 corrections), Q2M, M2M (all levels), M2L,
   L2L (all levels), L2P (with the diagonal term). */
int fabipb_b200_pass_times(void *ctx, const double *x, int reps, double *ms, int on_device);
/* the transposed operators, for adjoint solves (no counterpart in the
   reference): out = beta*out + alpha*K_part^T*lam, and
   y = alpha*(D - K)^T x + beta*y.  The transposed far field runs the FMM
   passes in reverse (Q2M^T = L2P-shaped, M2L over the transposed pair lists,
   L2L^T/M2M^T as shifts); the near field swaps the roles of the panels of a
   pair.  The first call builds the transposed lists (allocates). */
int fabipb_b200_apply_adjoint(void *ctx, int part, double alpha, const double *lam, double beta,
                              double *out, int on_device);
int fabipb_b200_matvec_adjoint(void *ctx, double alpha, const double *x, double beta, double *y,
                               int on_device);
/* right-hand side, 2N in tree order (setupRHS, src/fabipb.c:744):
   use_tree = 0 direct panel-charge sum, 1 charge-tree walk */
int fabipb_b200_rhs(void *ctx, int use_tree, double *rhs, int on_device);
/* raw solvation energy sum (before 2*pi*332.0716), panel-charge-tree walk
   (applyPanelChargeTreeEnergy, src/treecode.c:927) */
int fabipb_b200_energy(void *ctx, const double *sgm, double *raw, int on_device);
/* the same energy sum, allocating nothing: sgm (2N) and raw (1 double) are
   DEVICE pointers, the work is queued on the context's stream and *raw is
   ready when that stream reaches it.  Per-block partial sums go to a fixed
   128 KiB array in the library's device image (limit 4,194,304 panels); the
   charge tree must already exist (one fabipb_b200_energy or tree
   fabipb_b200_rhs call builds it).  Every call looks the array's address up
   in the current CUDA context (no allocation); the first call in a process
   may load the device image and should come before any stream capture.
   Calls in one CUDA context share the array: calls that overlap on the GPU
   race.  No counterpart in the reference, whose energy path allocates per
   call. */
int fabipb_b200_energy_noalloc(void *ctx, const double *sgm, double *raw);
/* gradients of the solvation energy with respect to the charges, surface
   fixed (no counterpart in the reference).  The energy here is the direct
   panel-charge sum E = e . sigma with e the energy weights (2N, pot slot
   eps dGk/dn - dG0/dn, dpdn slot G0 - Gk, times 2A and the quadrature
   weights); it equals fabipb_b200_energy with every charge-tree cluster
   opened.
   fabipb_b200_forward: direct RHS, GMRES from x0 = b with the current
   preconditioner (block LU set up when none is), E; keeps sigma.
   fabipb_b200_backward: the adjoint solve (D - K)^T lambda = e from
   lambda0 = e with its own Krylov basis, then per charge
   dE/dq_k = grad_energy * phi_k and dE/dr_k = grad_energy * q_k grad phi_k
   (dEdq: m values, dEdx: 3m, x y z per charge; either may be NULL). */
int fabipb_b200_energy_weights(void *ctx, double *e, int on_device);
int fabipb_b200_forward(void *ctx, int restart, int maxit, double tol, double *energy_raw, int *iters,
                        double *resid, int *info);
int fabipb_b200_backward(void *ctx, double grad_energy, int restart, int maxit, double tol, double *dEdq,
                         double *dEdx, int *iters, double *resid, int *info, int on_device);
/* preconditioner (src/precond_fmm.c): mode 2 block LU, 3 diagonal, -1 none */
int fabipb_b200_precond_setup(void *ctx, int mode);
int fabipb_b200_precond_apply(void *ctx, const double *b, double *x, int on_device);
/* restarted left-preconditioned GMRES on the device (src/gmres.c:153);
   x holds the initial guess on entry.  Returns info like the reference in
   *info (0 converged, 1 iteration limit, 2 breakdown). */
int fabipb_b200_solve(void *ctx, const double *b, double *x, int restart, int maxit,
                      double tol, int *iters, double *resid, int *info, int on_device);

#ifdef __cplusplus
}
#endif
#endif
