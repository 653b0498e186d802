// api.cu -- context lifecycle, composite operators and the plain-pointer C ABI
// declared in include/fabipb_b200.h.
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "context.cuh"
#include "quad.cuh"

namespace fb {

bool trace_enabled() {
  static const bool on = getenv("FABIPB_B200_TRACE") != nullptr;
  return on;
}

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

StageTimer::StageTimer(const char *sc, cudaStream_t s) : scope(sc), stream(s), on(trace_enabled()), t(0.0) {
  if (on) {
    cudaStreamSynchronize(stream);
    t = now_ms();
  }
}

void StageTimer::mark(const char *stage) {
  if (!on) return;
  cudaStreamSynchronize(stream);
  const double n = now_ms();
  fprintf(stderr, "[fabipb_b200] %s.%s %.3f ms\n", scope, stage, n - t);
  t = n;
}


static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

const char *get_error() { return g_err[0] ? g_err : "no error recorded"; }

bool init_quad_tables() {
  // Gauss-Legendre on [0,1], the published 15-decimal values the reference
  // tabulates in src/numQuad.c:221-294.
  static const double T[11][10] = {
      {0},
      {0.500000000000000},
      {0.211324865405187, 0.788675134594813},
      {0.112701665379258, 0.500000000000000, 0.887298334620742},
      {0.069431844202974, 0.330009478207572, 0.669990521792428, 0.930568155797026},
      {0.046910077030668, 0.230765344947158, 0.500000000000000, 0.769234655052841, 0.953089922969332},
      {0.033765242898424, 0.169395306766868, 0.380690406958402, 0.619309593041598, 0.830604693233132,
       0.966234757101576},
      {0.025446043828621, 0.129234407200303, 0.297077424311301, 0.500000000000000, 0.702922575688699,
       0.870765592799697, 0.974553956171379},
      {0.019855071751232, 0.101666761293187, 0.237233795041836, 0.408282678752175, 0.591717321247825,
       0.762766204958164, 0.898333238706813, 0.980144928248768},
      {0.015919880246187, 0.081984446336682, 0.193314283649705, 0.337873288298095, 0.500000000000000,
       0.662126711701904, 0.806685716350295, 0.918015553663318, 0.984080119753813},
      {0.013046735741414, 0.067468316655508, 0.160295215850488, 0.283302302935376, 0.425562830509184,
       0.574437169490816, 0.716697697064624, 0.839704784149512, 0.932531683344492, 0.986953264258586}};
  static const double W[11][10] = {
      {0},
      {1.000000000000000},
      {0.500000000000000, 0.500000000000000},
      {0.277777777777778, 0.444444444444444, 0.277777777777778},
      {0.173927422568727, 0.326072577431273, 0.326072577431273, 0.173927422568727},
      {0.118463442528095, 0.239314335249683, 0.284444444444444, 0.239314335249683, 0.118463442528095},
      {0.085662246189585, 0.180380786524070, 0.233956967286346, 0.233956967286346, 0.180380786524069,
       0.085662246189585},
      {0.064742483084435, 0.139852695744638, 0.190915025252560, 0.208979591836735, 0.190915025252559,
       0.139852695744638, 0.064742483084435},
      {0.050614268145188, 0.111190517226687, 0.156853322938944, 0.181341891689181, 0.181341891689181,
       0.156853322938944, 0.111190517226687, 0.050614268145188},
      {0.040637194180787, 0.090324080347429, 0.130305348201467, 0.156173538520002, 0.165119677500630,
       0.156173538520002, 0.130305348201468, 0.090324080347429, 0.040637194180787},
      {0.033335672154344, 0.074725674575290, 0.109543181257991, 0.134633359654998, 0.147762112357376,
       0.147762112357376, 0.134633359654998, 0.109543181257991, 0.074725674575290, 0.033335672154344}};
  FB_CUDA(cudaMemcpyToSymbol(c_tLeg, T, sizeof(T)));
  FB_CUDA(cudaMemcpyToSymbol(c_wLeg, W, sizeof(W)));
  return true;
}

// once per device (the current one): the default memory pool keeps freed memory
bool pool_keep_memory() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return true;
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
    set_error("no default memory pool on device %d", dev);
    return false;
  }
  uint64_t keep = UINT64_MAX;
  if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
    set_error("memory pool set-up failed on device %d", dev);
    return false;
  }
  done[dev] = true;
  return true;
}

Context::~Context() {
  free_charges(*this);
  free_precond(*this);
  free_adjoint(*this);
  arena.release();
  if (sideStream) cudaStreamDestroy(sideStream);
  if (farStream) cudaStreamDestroy(farStream);
  if (evFar) cudaEventDestroy(evFar);
  if (evFork) cudaEventDestroy(evFork);
  if (evJoin) cudaEventDestroy(evJoin);
  if (ownStream && stream) cudaStreamDestroy(stream);
}

bool build_panel_tree_device(Context &c, const double *vtxIn, const double *nrmIn, const double *areaIn);

// The panel tree on the device (tree_dev.cu), which also leaves the panels in
// tree order on the device; FABIPB_B200_HOST_TREE=1 builds it on the host
// threads instead (tree.cpp; the tests compare the two).
bool setup_geometry(Context &c, const double *vtx, const double *nrm, const double *area) {
  const int n = c.n;
  StageTimer tm("create", c.stream);
  const bool hostTree = getenv("FABIPB_B200_HOST_TREE") != nullptr;
  if (!hostTree) {
    if (!build_panel_tree_device(c, vtx, nrm, area)) return false;
    tm.mark("octree_device");
  } else {
    if (!build_panel_tree(c.pt, n, vtx, c.prm.depth, c.prm.height, c.prm.sep_ratio, c.prm.order,
                          c.prm.order_mom))
      return false;
    tm.mark("octree_host");
  }
  const PanelTree &pt = c.pt;
  if (hostTree) {   // the panels in tree order, gathered on host threads
    c.h_vtx.resize(9 * (size_t)n);
    c.h_nrm.resize(3 * (size_t)n);
    c.h_area.resize(n);
    auto gather = [&](int i0, int i1) {
      for (int i = i0; i < i1; i++) {
        int o = pt.order[i];
        memcpy(&c.h_vtx[9 * (size_t)i], &vtx[9 * (size_t)o], 9 * sizeof(double));
        memcpy(&c.h_nrm[3 * (size_t)i], &nrm[3 * (size_t)o], 3 * sizeof(double));
        c.h_area[i] = area[o];
      }
    };
    const int nth = n < 65536 ? 1 : (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int th = 1; th < nth; th++) pool.emplace_back(gather, (int)((long long)n * th / nth), (int)((long long)n * (th + 1) / nth));
    gather(0, (int)((long long)n / nth));
    for (auto &t : pool) t.join();
  }
  std::vector<int> leafOf(n);
  std::vector<double> leafCtr(3 * (size_t)pt.nLeaves);
  for (int L = 0; L < pt.nLeaves; L++) {
    for (int k = 0; k < pt.leafCount[L]; k++) leafOf[pt.leafStart[L] + k] = L;
    for (int k = 0; k < 3; k++) leafCtr[3 * (size_t)L + k] = pt.t.x[3 * (size_t)pt.leafCube[L] + k];
  }
  cudaStream_t s = c.stream;
  if (hostTree && (!c.arena.upload(&c.d_vtx, c.h_vtx, s) || !c.arena.upload(&c.d_nrm, c.h_nrm, s) ||
                   !c.arena.upload(&c.d_area, c.h_area, s)))
    return false;
  if (!c.arena.upload(&c.d_leafStart, pt.leafStart, s) ||
      !c.arena.upload(&c.d_leafCount, pt.leafCount, s) || !c.arena.upload(&c.d_leafOfPanel, leafOf, s) ||
      !c.arena.upload(&c.d_nearOff, pt.nearOff, s) || !c.arena.upload(&c.d_nearSrc, pt.nearSrc, s) ||
      !c.arena.upload(&c.d_leafCtr, leafCtr, s))
    return false;
  if (!c.arena.alloc_n(&c.d_x, 2 * (size_t)n) || !c.arena.alloc_n(&c.d_y, 2 * (size_t)n) ||
      !c.arena.alloc_n(&c.d_w, 2 * (size_t)n) || !c.arena.alloc_n(&c.d_nearOut, 2 * (size_t)n))
    return false;
  return true;
}

// pot = beta*pot + alpha*K_part*sgm (a direct context has no far part: its
// near field is every panel pair)
bool op_apply(Context &c, int part, double alpha, const double *sgm, double beta, double *pot, bool adjoint) {
  if (c.dense) part &= ~FABIPB_B200_FAR;
  if (part & FABIPB_B200_FAR) {
    if (!launch_far_upward(c, sgm, adjoint)) return false;
    if (!launch_l2p(c, alpha, beta, pot, nullptr, 0.0, 0.0, adjoint)) return false;
  } else if (beta != 1.0) {
    // scale pot by beta through L2P with alpha = 0 would still read lec;
    // a plain scale is cheaper
    if (beta == 0.0) {
      FB_CUDA(cudaMemsetAsync(pot, 0, 2 * (size_t)c.n * sizeof(double), c.stream));
    } else {
      extern bool scale_vec(Context &, double *, double, long long);
      if (!scale_vec(c, pot, beta, 2LL * c.n)) return false;
    }
  }
  if (part & FABIPB_B200_NEAR) {
    if (!launch_near(c, sgm, alpha, pot, adjoint)) return false;
  }
  return true;
}

// y = beta*y + s1*A.*x_pot, s2*A.*x_dpdn + add (the direct context's matvec:
// the diagonal of MtVmain, src/fabipb.c:1257-1265, plus its near term)
__global__ void direct_combine_kernel(int n, const double *__restrict__ area, const double *__restrict__ x,
                                      const double *__restrict__ add, double s1, double s2, double beta, double *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = area[i];
  const double y0 = beta == 0.0 ? 0.0 : beta * y[i], y1 = beta == 0.0 ? 0.0 : beta * y[i + n];
  y[i] = y0 + s1 * a * x[i] + add[i];
  y[i + n] = y1 + s2 * a * x[i + n] + add[i + n];
}

#ifndef FB_FAR_PRIORITY
#define FB_FAR_PRIORITY 1
#endif
// y = alpha*(D - K)x + beta*y, D = diag(s1*A, s2*A) (MtVmain); adjoint: (D - K^T)
bool op_matvec(Context &c, double alpha, const double *x, double beta, double *y, bool adjoint, bool fp64) {
  double s1 = (1.0 + c.epsilon) / 2.0 * alpha;
  double s2 = (1.0 + 1.0 / c.epsilon) / 2.0 * alpha;
  if (c.dense) {   // the direct operator: every panel pair through the near-field kernels
    if (!launch_near(c, x, -alpha, c.d_nearOut, adjoint, fp64, c.stream, false)) return false;
    direct_combine_kernel<<<ceil_div(c.n, 256), 256, 0, c.stream>>>(c.n, c.d_area, x, c.d_nearOut, s1, s2, beta, y);
    c.launches += 1;
    FB_CUDA(cudaGetLastError());
    return true;
  }
  // the near field on the side stream, into d_nearOut, beside the far passes
  FB_CUDA(cudaEventRecord(c.evFork, c.stream));
  FB_CUDA(cudaStreamWaitEvent(c.sideStream, c.evFork, 0));
  if (!launch_near(c, x, -alpha, c.d_nearOut, adjoint, fp64, c.sideStream, false)) return false;
  FB_CUDA(cudaEventRecord(c.evJoin, c.sideStream));
#if FB_FAR_PRIORITY
  // the far passes on the high-priority stream (the launch helpers use c.stream)
  FB_CUDA(cudaStreamWaitEvent(c.farStream, c.evFork, 0));
  cudaStream_t user = c.stream;
  c.stream = c.farStream;
  const bool farOk = launch_far_upward(c, x, adjoint, nullptr, fp64);
  c.stream = user;
  if (!farOk) return false;
  FB_CUDA(cudaEventRecord(c.evFar, c.farStream));
  FB_CUDA(cudaStreamWaitEvent(c.stream, c.evFar, 0));
#else
  if (!launch_far_upward(c, x, adjoint, nullptr, fp64)) return false;
#endif
  FB_CUDA(cudaStreamWaitEvent(c.stream, c.evJoin, 0));
  if (!launch_l2p(c, -alpha, beta, y, x, s1, s2, adjoint, c.d_nearOut, fp64)) return false;
  return true;
}

__global__ void scale_kernel(double *v, double a, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] *= a;
}

bool scale_vec(Context &c, double *v, double a, long long n) {
  c.launches += 1;
  scale_kernel<<<ceil_div(n, 256), 256, 0, c.stream>>>(v, a, n);
  FB_CUDA(cudaGetLastError());
  return true;
}

int create_context(const fabipb_b200_params *p, int n, const double *vtx, const double *normal,
                   const double *area, bool dense, void **out) {
  if (out) *out = nullptr;
  if (p == nullptr || vtx == nullptr || normal == nullptr || area == nullptr || out == nullptr || n <= 0) {
    set_error("fabipb_b200_create: invalid arguments");
    return 0;
  }
  auto t0 = std::chrono::steady_clock::now();
  Context *c = new Context();
  c->prm = *p;
  c->n = n;
  c->epsilon = p->eps2 / p->eps1;
  c->mixed = (p->precision == FABIPB_B200_MIXED);
  c->device = p->device;
  c->dense = dense;
  bool ok = true;
  if (cudaSetDevice(p->device) != cudaSuccess) {
    set_error("cudaSetDevice(%d) failed", p->device);
    ok = false;
  }
  if (ok && cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cudaStreamCreate failed");
    ok = false;
  }
  c->ownStream = ok;
  int prLeast = 0, prGreatest = 0;
  if (ok) cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest);
  if (ok && (cudaStreamCreateWithFlags(&c->sideStream, cudaStreamNonBlocking) != cudaSuccess ||
             cudaStreamCreateWithPriority(&c->farStream, cudaStreamNonBlocking, prGreatest) != cudaSuccess ||
             cudaEventCreateWithFlags(&c->evFork, cudaEventDisableTiming) != cudaSuccess ||
             cudaEventCreateWithFlags(&c->evJoin, cudaEventDisableTiming) != cudaSuccess ||
             cudaEventCreateWithFlags(&c->evFar, cudaEventDisableTiming) != cudaSuccess)) {
    set_error("stream/event creation failed");
    ok = false;
  }
  StageTimer tm("create", c->stream);
  ok = ok && init_quad_tables();
  ok = ok && setup_geometry(*c, vtx, normal, area);
  tm.mark("tree_and_geometry");
  ok = ok && setup_near(*c);
  tm.mark("near_setup");
  ok = ok && setup_fmm(*c);
  tm.mark("fmm_setup");
  // the geometry-only tables of the adjoint operator (the transposed special
  // pairs and M2L lists) and, in a mixed context, the FP64 near-field records
  // of the refinement residuals: built here, once, so that no solve, backward
  // pass or refinement pays for them on its first call
  ok = ok && setup_near_adjoint(*c);
  tm.mark("near_adjoint");
  ok = ok && setup_m2l_adjoint(*c);
  tm.mark("m2l_adjoint");
  ok = ok && (!c->mixed || setup_near_fp64(*c));
  tm.mark("near_fp64");
  if (ok && cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("setup kernels failed: %s", cudaGetErrorString(cudaGetLastError()));
    ok = false;
  }
  if (!ok) {
    std::string keep = get_error();
    delete c;
    set_error("%s", keep.c_str());
    return 0;
  }
  c->setupSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  *out = c;
  return 1;
}

}  // namespace fb

using namespace fb;

static bool valid_ctx(void *ctx) {
  if (ctx == nullptr) {
    set_error("null context");
    return false;
  }
  return true;
}

// Run `fn` on device vectors; for host pointers copy in/out around it.
template <typename F>
static int with_vectors(Context *c, const double *in, double *inout, bool readOut, int on_device, F fn) {
  cudaSetDevice(c->device);
  const size_t bytes = 2 * (size_t)c->n * sizeof(double);
  if (on_device) {
    if (!fn(in, inout)) return 0;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
      set_error("kernel failure: %s", cudaGetErrorString(cudaGetLastError()));
      return 0;
    }
    return 1;
  }
  if (in && cudaMemcpyAsync(c->d_x, in, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
    set_error("host-to-device copy failed");
    return 0;
  }
  if (readOut && cudaMemcpyAsync(c->d_y, inout, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
    set_error("host-to-device copy failed");
    return 0;
  }
  if (!fn(in ? c->d_x : nullptr, c->d_y)) return 0;
  if (cudaMemcpyAsync(inout, c->d_y, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) {
    set_error("device-to-host copy failed");
    return 0;
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("kernel failure: %s", cudaGetErrorString(cudaGetLastError()));
    return 0;
  }
  return 1;
}

extern "C" {

void fabipb_b200_default_params(fabipb_b200_params *p) {
  p->order = 3;
  p->order_mom = 0;
  p->depth = 5;
  p->height = 2;
  p->quad_order = 1;
  p->sep_ratio = 0.8;
  p->kappa = 0.1257;
  p->eps1 = 1.0;
  p->eps2 = 80.0;
  p->rhs_theta = 0.8;
  p->energy_theta = 0.8;
  p->charge_order = 0;
  p->precision = FABIPB_B200_MIXED;
  p->device = 0;
}

const char *fabipb_b200_last_error(void) { return get_error(); }

int fabipb_b200_create(const fabipb_b200_params *p, int n, const double *vtx, const double *normal,
                       const double *area, void **out) {
  return create_context(p, n, vtx, normal, area, false, out);
}

int fabipb_b200_create_direct(const fabipb_b200_params *p, int n, const double *vtx, const double *normal,
                              const double *area, void **out) {
  return create_context(p, n, vtx, normal, area, true, out);
}

void fabipb_b200_destroy(void *ctx) {
  if (ctx == nullptr) return;
  Context *c = (Context *)ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete c;
}

int fabipb_b200_set_stream(void *ctx, void *stream) {
  if (!valid_ctx(ctx)) return 0;
  Context *c = (Context *)ctx;
  if (c->ownStream && c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  c->ownStream = false;
  c->stream = (cudaStream_t)stream;
  return 1;
}

int fabipb_b200_info_get(void *ctx, fabipb_b200_info *o) {
  if (!valid_ctx(ctx) || o == nullptr) return 0;
  Context *c = (Context *)ctx;
  o->panels = c->n;
  o->leaves = c->pt.nLeaves;
  o->near_pairs = (int)c->pt.nearSrc.size();
  o->m2l_pairs = (int)c->pt.m2lSrc.size();
  o->cubes = c->pt.nFmm;
  o->max_order = c->P;
  o->leaf_order = c->leafOrder;
  o->max_leaf = c->maxLeaf;
  o->near_panel_pairs = c->nearPanelPairs;
  o->special_pairs = c->nSpecial;
  o->setup_seconds = c->setupSeconds;
  o->device_bytes = (double)c->arena.bytes;
  return 1;
}

long long fabipb_b200_launch_count(void *ctx) {
  if (ctx == nullptr) return -1;
  return ((Context *)ctx)->launches;
}

int fabipb_b200_panel_order(void *ctx, int *order) {
  if (!valid_ctx(ctx) || order == nullptr) return 0;
  Context *c = (Context *)ctx;
  memcpy(order, c->pt.order.data(), (size_t)c->n * sizeof(int));
  return 1;
}

int fabipb_b200_leaf_layout(void *ctx, int *start, int *count) {
  if (!valid_ctx(ctx)) return 0;
  Context *c = (Context *)ctx;
  memcpy(start, c->pt.leafStart.data(), c->pt.leafStart.size() * sizeof(int));
  memcpy(count, c->pt.leafCount.data(), c->pt.leafCount.size() * sizeof(int));
  return 1;
}

int fabipb_b200_near_pairs(void *ctx, int *src, int *dst) {
  if (!valid_ctx(ctx)) return 0;
  Context *c = (Context *)ctx;
  memcpy(src, c->pt.nearSrc.data(), c->pt.nearSrc.size() * sizeof(int));
  memcpy(dst, c->pt.nearDst.data(), c->pt.nearDst.size() * sizeof(int));
  return 1;
}

int fabipb_b200_m2l_pairs(void *ctx, int *src, int *dst) {
  if (!valid_ctx(ctx)) return 0;
  Context *c = (Context *)ctx;
  memcpy(src, c->pt.m2lPairSrc.data(), c->pt.m2lPairSrc.size() * sizeof(int));
  memcpy(dst, c->pt.m2lPairDst.data(), c->pt.m2lPairDst.size() * sizeof(int));
  return 1;
}

int fabipb_b200_cube_data(void *ctx, int *level, double *ctr4) {
  if (!valid_ctx(ctx)) return 0;
  Context *c = (Context *)ctx;
  for (int f = 0; f < c->pt.nFmm; f++) {
    int cc = c->pt.fmmCube[f];
    level[f] = c->pt.t.level[cc];
    for (int k = 0; k < 3; k++) ctr4[4 * f + k] = c->pt.t.x[3 * (size_t)cc + k];
    ctr4[4 * f + 3] = c->pt.t.rad[cc];
  }
  return 1;
}

int fabipb_b200_apply(void *ctx, int part, double alpha, const double *sgm, double beta, double *pot,
                      int on_device) {
  if (!valid_ctx(ctx) || sgm == nullptr || pot == nullptr) return 0;
  Context *c = (Context *)ctx;
  if (part < 1 || part > 3) {
    set_error("fabipb_b200_apply: part must be NEAR, FAR or ALL");
    return 0;
  }
  return with_vectors(c, sgm, pot, beta != 0.0, on_device, [&](const double *x, double *y) {
    return op_apply(*c, part, alpha, x, beta, y);
  });
}

int fabipb_b200_matvec(void *ctx, double alpha, const double *x, double beta, double *y, int on_device) {
  if (!valid_ctx(ctx) || x == nullptr || y == nullptr) return 0;
  Context *c = (Context *)ctx;
  return with_vectors(c, x, y, beta != 0.0, on_device, [&](const double *xd, double *yd) {
    return op_matvec(*c, alpha, xd, beta, yd);
  });
}

int fabipb_b200_pass_times(void *ctx, const double *x, int reps, double *ms, int on_device) {
  if (!valid_ctx(ctx) || x == nullptr || ms == nullptr || reps < 1) {
    set_error("fabipb_b200_pass_times: invalid arguments");
    return 0;
  }
  Context *c = (Context *)ctx;
  cudaEvent_t ev[7];
  for (int i = 0; i < 7; i++) cudaEventCreate(&ev[i]);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  cudaSetDevice(c->device);
  bool ok = true;
  const double *xd = x;
  if (ok && !on_device) {
    ok = cudaMemcpyAsync(c->d_x, x, 2 * (size_t)c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream) ==
         cudaSuccess;
    xd = c->d_x;
  }
  for (int r = 0; ok && r < reps; r++) {
    cudaEventRecord(ev[0], c->stream);
    ok = launch_near(*c, xd, -1.0, c->d_y);
    cudaEventRecord(ev[1], c->stream);
    ok = ok && launch_far_upward(*c, xd, false, ev + 2);
    ok = ok && launch_l2p(*c, -1.0, 1.0, c->d_y, xd, 1.0, 1.0);
    cudaEventRecord(ev[6], c->stream);
    if (ok) ok = cudaEventSynchronize(ev[6]) == cudaSuccess;
    for (int i = 0; ok && i < 6; i++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      acc[i] += t;
    }
  }
  for (int i = 0; i < 7; i++) cudaEventDestroy(ev[i]);
  if (!ok) {
    set_error("pass timing failed: %s", get_error());
    return 0;
  }
  for (int i = 0; i < 6; i++) ms[i] = acc[i] / reps;
  return 1;
}

int fabipb_b200_solve_refined(void *ctx, const double *b, double *x, int restart, int maxit, double tol_inner,
                              double tol, int max_outer, int *outer, int *iters, double *resid, int *info,
                              int on_device) {
  if (!valid_ctx(ctx) || b == nullptr || x == nullptr || restart < 1 || maxit < 1 || max_outer < 0) {
    set_error("fabipb_b200_solve_refined: invalid arguments");
    return 0;
  }
  Context *c = (Context *)ctx;
  int ou = 0, it = 0, inf = 0;
  double res = 0.0;
  StageTimer tm("solve", c->stream);
  int ok = with_vectors(c, b, x, true, on_device, [&](const double *bd, double *xd) {
    return refined_solve(*c, bd, xd, restart, maxit, tol_inner, tol, max_outer, &ou, &it, &res, &inf);
  });
  tm.mark("refined");
  if (outer) *outer = ou;
  if (iters) *iters = it;
  if (resid) *resid = res;
  if (info) *info = inf;
  return ok;
}

int fabipb_b200_apply_adjoint(void *ctx, int part, double alpha, const double *lam, double beta, double *out,
                              int on_device) {
  if (!valid_ctx(ctx) || lam == nullptr || out == nullptr) return 0;
  Context *c = (Context *)ctx;
  if (part < 1 || part > 3) {
    set_error("fabipb_b200_apply_adjoint: part must be NEAR, FAR or ALL");
    return 0;
  }
  return with_vectors(c, lam, out, beta != 0.0, on_device, [&](const double *x, double *y) {
    return op_apply(*c, part, alpha, x, beta, y, true);
  });
}

int fabipb_b200_matvec_adjoint(void *ctx, double alpha, const double *x, double beta, double *y, int on_device) {
  if (!valid_ctx(ctx) || x == nullptr || y == nullptr) return 0;
  Context *c = (Context *)ctx;
  return with_vectors(c, x, y, beta != 0.0, on_device, [&](const double *xd, double *yd) {
    return op_matvec(*c, alpha, xd, beta, yd, true);
  });
}

}  // extern "C"

extern "C" {

int fabipb_b200_set_charges(void *ctx, int m, const double *pos, const double *q) {
  if (!valid_ctx(ctx) || m <= 0 || pos == nullptr || q == nullptr) {
    set_error("fabipb_b200_set_charges: invalid arguments");
    return 0;
  }
  Context *c = (Context *)ctx;
  cudaSetDevice(c->device);
  free_adjoint(*c);   // a forward solve of the old charges is void
  if (!setup_charges(*c, m, pos, q)) return 0;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("charge setup failed: %s", cudaGetErrorString(cudaGetLastError()));
    return 0;
  }
  return 1;
}

int fabipb_b200_rhs(void *ctx, int use_tree, double *rhs, int on_device) {
  if (!valid_ctx(ctx) || rhs == nullptr) return 0;
  Context *c = (Context *)ctx;
  StageTimer tm("rhs", c->stream);
  int ok = with_vectors(c, nullptr, rhs, false, on_device, [&](const double *, double *y) {
    return launch_rhs(*c, use_tree, y);
  });
  tm.mark(use_tree ? "tree" : "direct");
  return ok;
}

int fabipb_b200_energy(void *ctx, const double *sgm, double *raw, int on_device) {
  if (!valid_ctx(ctx) || sgm == nullptr || raw == nullptr) return 0;
  Context *c = (Context *)ctx;
  cudaSetDevice(c->device);
  const double *d = sgm;
  if (!on_device) {
    if (cudaMemcpyAsync(c->d_x, sgm, 2 * (size_t)c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess) {
      set_error("host-to-device copy failed");
      return 0;
    }
    d = c->d_x;
  }
  if (!launch_energy(*c, d, raw)) return 0;
  return 1;
}

int fabipb_b200_precond_setup(void *ctx, int mode) {
  if (!valid_ctx(ctx)) return 0;
  Context *c = (Context *)ctx;
  cudaSetDevice(c->device);
  if (!precond_setup(*c, mode)) return 0;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("preconditioner setup failed: %s", cudaGetErrorString(cudaGetLastError()));
    return 0;
  }
  return 1;
}

int fabipb_b200_precond_apply(void *ctx, const double *b, double *x, int on_device) {
  if (!valid_ctx(ctx) || b == nullptr || x == nullptr) return 0;
  Context *c = (Context *)ctx;
  return with_vectors(c, b, x, false, on_device, [&](const double *bd, double *xd) {
    return precond_apply(*c, bd, xd);
  });
}

int fabipb_b200_solve(void *ctx, const double *b, double *x, int restart, int maxit, double tol, int *iters,
                      double *resid, int *info, int on_device) {
  if (!valid_ctx(ctx) || b == nullptr || x == nullptr || restart < 1 || maxit < 1) {
    set_error("fabipb_b200_solve: invalid arguments");
    return 0;
  }
  Context *c = (Context *)ctx;
  int it = 0, inf = 0;
  double res = 0.0;
  StageTimer tm("solve", c->stream);
  int ok = with_vectors(c, b, x, true, on_device, [&](const double *bd, double *xd) {
    return gmres_solve(*c, bd, xd, restart, maxit, tol, &it, &res, &inf);
  });
  tm.mark("gmres");
  if (iters) *iters = it;
  if (resid) *resid = res;
  if (info) *info = inf;
  return ok;
}

}  // extern "C"
