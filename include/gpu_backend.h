/*
 * gpu_backend.h -- the reference's GPU plugin ABI, implemented by
 * libfabipb_b200.so.  The signatures are those of include/gpu_backend.h:12-47
 * of the reference (each line below names the one it replaces); a host built
 * from the reference sources links this library instead of its
 * src/gpu_backend_cuda.cu and runs unchanged.
 *
 * Convention (reference src/gpu_backend_cuda.cu:306-326): 1 = handled,
 * 0 = not handled with a message in the last-error strings.  Vectors are host
 * arrays of length 2N indexed by pnl->idx.  The device state is cached per
 * `struct ssystem *` and rebuilt when a different system is passed.
 *
 * Arithmetic: FP64 by default, as the reference backend; the environment
 * variable FABIPB_B200_PRECISION=mixed selects the FP32 near-field P2P.
 */
#ifndef FABIPB_B200_GPU_BACKEND_H
#define FABIPB_B200_GPU_BACKEND_H

struct panel;
struct ssystem;

#ifdef __cplusplus
extern "C" {
#endif

/* gpu_backend.h:12 -- 1 when a CUDA device is present */
int gpuBackendAvailable(void);
/* gpu_backend.h:13-14 -- last failure messages */
const char *gpuNearfieldLastError(void);
const char *gpuM2LLastError(void);
/* gpu_backend.h:15 -- pot += alpha * K_near * sgm */
int gpuNearfieldApply(struct ssystem *sys, double alpha, const double *sgm, double *pot);
/* gpu_backend.h:16 -- pot = beta*pot + alpha * K_dense * sgm (every pair) */
int gpuDirectApply(struct ssystem *sys, double alpha, double beta, const double *sgm, double *pot);
/* gpu_backend.h:17 -- interaction pass.  After gpuQ2MApply in the same
   matvec the expansions already live on the device and this returns 1
   without touching the host cubes; otherwise it reads the host moments and
   writes the host local expansions */
int gpuM2LApply(struct ssystem *sys);
/* gpu_backend.h:18 -- leaf moments.  Runs Q2M, M2M, M2L and L2L on the
   device and leaves the host moments zero (so the host's M2M/L2L loops add
   nothing) */
int gpuQ2MApply(struct ssystem *sys, const double *sgm);
/* gpu_backend.h:19 -- pot = beta*pot + alpha * L2P(local expansions) */
int gpuL2PApply(struct ssystem *sys, double alpha, double beta, double *pot);
/* gpu_backend.h:20-21 -- free the cached device state */
void gpuReleaseMatvecCaches(void);
void gpuReleaseChargeTreeCache(void);
/* gpu_backend.h:22 -- direct right-hand side, sgm = fac * sum_charges ... */
int gpuSetupRHS(struct ssystem *sys, int qOrder, double fac, double *sgm);
/* gpu_backend.h:28 -- raw panel-tree solvation energy */
int gpuPanelChargeTreeEnergy(struct ssystem *sys, const double *sgm, double *pot);
/* gpu_backend.h:29-30 -- eps1 * sum(rhs0*sgm1 - rhs1*sgm0) */
int gpuRhsReuseCoulombDot(struct ssystem *sys, const double *rhs, const double *sgm, double *dot);
/* gpu_backend.h:31-32 -- Coulomb dot + screened-only tree energy */
int gpuRhsReusePanelChargeTreeEnergy(struct ssystem *sys, const double *rhs, const double *sgm,
                                     double *pot);
/* gpu_backend.h:34 -- charge-tree right-hand side */
int gpuChargeTreeRHS(struct ssystem *sys, int qOrder, double fac, double *sgm);
/* gpu_backend.h:41-44 -- one-point disjoint coefficients of listed pairs
   (X = pairDst[t], Y = pairSrc[t], both pnl->idx); non-disjoint pairs are
   left untouched */
int gpuBuildPrecondPairsBatched(struct ssystem *sys, const int *pairSrc, const int *pairDst,
                                long long nPairs, double *k0, double *k1, double *k2, double *k3);
/* gpu_backend.h:45-47 -- negated disjoint coefficients written into one
   preconditioner block (thread safe) */
int gpuBuildPrecondDisjointBlock(struct panel **panels, int nPanels, const int *dstLocal,
                                 const int *srcLocal, int nPairs, double *block);

#ifdef __cplusplus
}
#endif
#endif
