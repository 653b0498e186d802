// context.cuh -- the device-resident state of one surface mesh.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/fabipb_b200.h"
#include "common.cuh"
#include "tree.hpp"

namespace fb {

struct ChargeTreeDev;
struct PrecondDev;
struct AdjointDev;
struct GraphCache;

struct Context {
  fabipb_b200_params prm{};
  double epsilon = 80.0;  // eps2 / eps1
  int device = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  DevArena arena;

  // ---- panels (tree order) and tree ----------------------------------
  PanelTree pt;
  int n = 0;
  std::vector<double> h_vtx, h_nrm, h_area;  // tree order (host copy)
  double *d_vtx = nullptr, *d_nrm = nullptr, *d_area = nullptr;
  int *d_leafStart = nullptr, *d_leafCount = nullptr, *d_leafOfPanel = nullptr;
  int *d_nearOff = nullptr, *d_nearSrc = nullptr;
  double *d_leafCtr = nullptr;             // 3 per leaf: enclosing-box centre
  int nWork = 0;                           // near-field warp tasks
  int2 *d_work = nullptr;                  // (leaf, 32-target group)
  long long nearPanelPairs = 0;
  int maxLeaf = 0;

  // ---- near field -------------------------------------------------------
  bool mixed = false;                      // FP32 P2P when true
  void *d_tgtP = nullptr, *d_tgtN = nullptr;   // T4: {rel pos, area}, {normal, 0}
  void *d_srcA = nullptr, *d_srcB = nullptr;   // T4: {rel pos, A*s_dpdn}, {normal, A*s_pot}
  long long nSpecial = 0;
  int *d_spOff = nullptr, *d_spSrc = nullptr;  // CSR by destination panel
  double4 *d_spK = nullptr;                    // exact minus one-point coefficient
  double4 *d_spKT = nullptr;                   // the same for the transposed operator
  void *d_tgtP64 = nullptr, *d_tgtN64 = nullptr;   // FP64 records of a mixed context (refinement residuals)
  // the symmetric near field: unordered leaf pairs (register leaf, tile leaf, scratch offsets),
  // per near-list entry its scratch offset (-1: the ordered kernel computes it); scratch and
  // records in the context's near-field precision (2 and 4 floats or doubles per entry)
  int nSymTasks = 0;
  int nSym32 = 0;                              // the first nSym32 tasks are 32-wide, the rest half-warp
  long long symPanelPairs = 0;                 // unordered panel pairs of those leaf pairs
  int4 *d_symTask = nullptr;
  int *d_symOff = nullptr;
  void *d_symScr = nullptr;
  void *d_symA = nullptr, *d_symB = nullptr;   // records {position, A*sigma_dpdn}, {normal, A*sigma_pot}
  void *d_srcA64 = nullptr, *d_srcB64 = nullptr;

  // ---- FMM ----------------------------------------------------------
  int P = 0, NM = 0;                       // max order, nmom(max order)
  int leafOrder = 0, NMleaf = 0;
  double *d_Q0 = nullptr, *d_Q1 = nullptr; // [NMleaf][n]: moments, noments
  float *d_Q0F = nullptr, *d_Q1F = nullptr; // their FP32 copies (mixed contexts)
  double *d_cubeCtr = nullptr;             // 3 per FMM cube
  int *d_m2lOff = nullptr, *d_m2lSrc = nullptr;
  int *d_fmmParent = nullptr;              // parent FMM index (or -1)
  int *d_leafFmm = nullptr;                // leaf -> FMM index
  double *d_mom = nullptr;                 // [2][nFmm][NM]  pot, dpdn
  double *d_lec = nullptr;                 // [4][nFmm][NM]
  std::vector<int> h_m2lDst;               // destination cubes with a list
  int *d_m2lDst = nullptr;
  int *d_lstOff = nullptr, *d_lst = nullptr;   // (beta, alpha+beta, |beta|) per alpha
  int *d_mOff = nullptr, *d_mLst = nullptr;    // (alpha-k, k) per alpha
  int *d_kidFirst = nullptr, *d_kidCount = nullptr;  // FMM indices of the children
  int *d_ordM2L = nullptr;                     // per FMM cube
  int nConvList = 0;                           // entries of d_lst
  std::vector<int> h_lstOff, h_mOff;           // host copies of the list offsets
  long long nM2LPairs = 0;
  double2 *d_m2lTens = nullptr;                // [nMom][pairs] (D G0, D Gk) per M2L pair
  float2 *d_m2lTensF = nullptr;                // the same in FP32 (mixed contexts, orders <= 5)
  float2 *d_momF2 = nullptr;                   // FP32 (pot, dpdn) rows of the M2L input, bulk-copy staging
  int momF2Stride = 0;                         // float2 entries per row (a 16-byte multiple)
  // transposed M2L lists (adjoint operator)
  bool m2lAdjReady = false;
  std::vector<int> h_m2lDstT;
  int *d_m2lDstT = nullptr, *d_m2lOffT = nullptr, *d_m2lSrcT = nullptr, *d_m2lPairT = nullptr;

  // ---- scratch vectors for host-pointer calls ------------------------
  double *d_x = nullptr, *d_y = nullptr, *d_w = nullptr;
  double *d_refR = nullptr, *d_refD = nullptr, *d_refZ = nullptr;   // iterative refinement (first use)
  // the matvec runs the near field on a second stream beside the far passes
  cudaStream_t sideStream = nullptr;
  // the far passes on a high-priority stream, so that their (short, latency-
  // bound) blocks are dispatched ahead of the near field's as SMs free up
  cudaStream_t farStream = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr, evFar = nullptr;
  double *d_nearOut = nullptr;             // 2N: the near-field term of the current matvec

  // ---- charges, RHS, energy -------------------------------------------
  std::vector<int> chargeOrders;           // per-level charge-tree order (host policy)
  double rhsFac = 0.0;                     // RHS scale override (0: 1/(4 pi eps1))
  bool dense = false;                      // near field over every leaf pair (direct mode)
  int nChar = 0;
  std::vector<double> h_pos, h_chr;
  ChargeTreeDev *ct = nullptr;

  // ---- preconditioner and GMRES ---------------------------------------
  PrecondDev *pc = nullptr;
  AdjointDev *adj = nullptr;               // forward/backward state (gradients)
  GraphCache *graphs = nullptr;

  double setupSeconds = 0.0;
  long long launches = 0;                  // kernels launched by this context
  ~Context();
};

// setup pieces (each returns false with the error recorded)
bool setup_geometry(Context &c, const double *vtx, const double *nrm, const double *area);
bool setup_near(Context &c);
bool setup_fmm(Context &c);
bool setup_charges(Context &c, int m, const double *pos, const double *q);

// device operators on device vectors (stream-ordered, no synchronisation)
// near:  out += coef * K_near * sgm
// (fp64: the FP64 P2P in a mixed context, for refinement residuals; stream:
// the stream to launch on, default the context's; accumulate = false writes
// out = coef * K_near * sgm)
bool launch_near(Context &c, const double *sgm, double coef, double *out, bool adjoint = false, bool fp64 = false,
                 cudaStream_t stream = nullptr, bool accumulate = true);
// upward pass + interaction + downward pass: leaves local expansions in d_lec
// (adjoint: the transposed far operator's upward half, see fmm.cu)
// (marks: 4 events recorded after Q2M, M2M, M2L and L2L, for pass timing)
// (fp64: the FP64 interaction also in a mixed context, for refinement residuals)
bool launch_far_upward(Context &c, const double *sgm, bool adjoint = false, cudaEvent_t *marks = nullptr,
                       bool fp64 = false);
// L2P: out = beta*out + alpha*far + diag*(area .* x) (diag part optional)
// (addend: a vector added to out, the near field computed beside the far passes)
// (fp64: the FP64 leaf matrices also in a mixed context, for refinement residuals)
bool launch_l2p(Context &c, double alpha, double beta, double *out, const double *diagX,
                double s1, double s2, bool adjoint = false, const double *addend = nullptr, bool fp64 = false);
bool launch_m2l_only(Context &c, bool adjoint = false, bool fp64 = false);
bool launch_rhs(Context &c, int useTree, double *rhs);
bool launch_energy(Context &c, const double *sgm, double *raw_host);
bool precond_setup(Context &c, int mode);
// (adjoint: the transposed preconditioner and operator, for A^T lambda = e)
bool precond_apply(Context &c, const double *b, double *x, bool adjoint = false);
// (steps: the Arnoldi steps actually taken; *iters follows the reference and
// keeps maxit when x already meets tol)
bool gmres_solve(Context &c, const double *b, double *x, int restart, int maxit, double tol,
                 int *iters, double *resid, int *info, bool adjoint = false, int *steps = nullptr);
// iterative refinement: FP64 residuals, corrections by GMRES on the context's operator
bool refined_solve(Context &c, const double *b, double *x, int restart, int maxit, double tolInner, double tol,
                   int maxOuter, int *outer, int *iters, double *resid, int *info);
void free_charges(Context &c);
void free_precond(Context &c);
void free_adjoint(Context &c);
bool dot_to_host(Context &c, long long n, const double *x, const double *y, double *out);

// create a context (dense = every leaf pair is near: the direct operator)
int create_context(const fabipb_b200_params *p, int n, const double *vtx, const double *nrm, const double *area,
                   bool dense, void **out);

// composite operators (device vectors)
// (adjoint: the transposed operator K^T, and (D - K)^T)
bool op_apply(Context &c, int part, double alpha, const double *sgm, double beta, double *pot, bool adjoint = false);
bool op_matvec(Context &c, double alpha, const double *x, double beta, double *y, bool adjoint = false,
               bool fp64 = false);

}  // namespace fb
