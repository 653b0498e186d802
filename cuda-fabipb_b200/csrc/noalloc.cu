// noalloc.cu -- the solvation-energy reduction without any device allocation.
//
// fabipb_b200_energy keeps its per-block partial sums in a buffer that the
// charge tree allocates on first use, and copies the result to the host.
// Some callers cannot let a library allocate device memory while they run:
// a serving process that hands the whole GPU to its own pool allocator at
// start-up (a framework caching allocator, a fixed arena sized for the largest
// mesh) must not see cudaMalloc/cudaFree from a library in the middle of its
// own work, since an allocation there can fail or fragment the pool, and a
// caller that keeps every operand on the device wants no host round trip.
// fabipb_b200_energy_noalloc serves them: device input, device output, and
// its scratch is a fixed array in the library's own device image.
//
// The scratch: g_energyScratch, kNoAllocMaxBlocks doubles (128 KiB), one per
// 256-panel block of the tree walk, so surfaces of up to 4,194,304 panels.
// Every GPU that loads this library holds the array until the process exits.
// The array's name in host code is only a host-side stand-in, so its device
// address is looked up with cudaGetSymbolAddress, which allocates nothing, on
// every call with the context's device current: the address always belongs to
// the CUDA context current on the calling thread (after a cudaDeviceReset, or
// under another context, the module and its array are loaded anew there).  The
// first call in a process may load the library's device image; make it before
// any stream capture.  Each CUDA context holds its own copy of the array; all
// calls in one context share it, and it keeps the last call's partial sums.
// Each block of the walk writes its entry before the final sum reads it, so
// nothing needs clearing.  Calls in one context that overlap on the GPU (two
// streams, two library contexts on one device) race on the array: serialise
// them.

namespace fb {

constexpr int kNoAllocMaxBlocks = 16384;
static __device__ __align__(256) double g_energyScratch[kNoAllocMaxBlocks];

// the array's device address in the current context (device `device`)
static double *noalloc_scratch(int device) {
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != device) {
    set_error("scratch look-up: device %d is not current", device);
    return nullptr;
  }
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_energyScratch);
  if (e != cudaSuccess || p == nullptr) {
    set_error("scratch look-up on device %d failed: %s", device, cudaGetErrorString(e));
    return nullptr;
  }
  return (double *)p;
}

}  // namespace fb

extern "C" int fabipb_b200_energy_noalloc(void *ctx, const double *sgm, double *raw) {
  if (!valid_ctx(ctx)) return 0;
  if (sgm == nullptr || raw == nullptr) {
    set_error("fabipb_b200_energy_noalloc: null vector");
    return 0;
  }
  Context *c = (Context *)ctx;
  if (c->ct == nullptr || c->nChar <= 0 || !c->ct->built) {
    set_error("fabipb_b200_energy_noalloc: no charge tree yet (fabipb_b200_set_charges, then one "
              "fabipb_b200_energy or tree fabipb_b200_rhs call builds it)");
    return 0;
  }
  const long long blocks = ceil_div((long long)c->n, 256);
  if (blocks > kNoAllocMaxBlocks) {
    set_error("fabipb_b200_energy_noalloc: %d panels above the limit of %lld (fixed scratch of %d blocks)", c->n,
              (long long)kNoAllocMaxBlocks * 256, kNoAllocMaxBlocks);
    return 0;
  }
  if (cudaSetDevice(c->device) != cudaSuccess) {
    set_error("fabipb_b200_energy_noalloc: cannot select device %d", c->device);
    return 0;
  }
  double *scratch = noalloc_scratch(c->device);
  if (scratch == nullptr) return 0;
  // the same walk as fabipb_b200_energy (mode 1), partial sums into the fixed array
  FB_DISPATCH_WALK(c->P, *c, 1, sgm, nullptr, scratch);
  sum_partials_kernel<<<1, kSumThreads, 0, c->stream>>>((int)blocks, scratch, raw);
  c->launches += 2;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("fabipb_b200_energy_noalloc: launch failed: %s", cudaGetErrorString(e));
    return 0;
  }
  return 1;
}
