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
// Its device address is looked up once per device (cudaGetSymbolAddress with
// that device current) by the first call on that device; that first call
// should therefore come before any stream capture.  Every call on a device
// shares the one array, which keeps the last call's partial sums; each block
// of the walk writes its entry before the final sum reads it, so nothing needs
// clearing.  Calls that overlap on the GPU (two streams, two contexts on one
// device) race on the array: serialise them.

#include <mutex>

namespace fb {

constexpr int kNoAllocMaxBlocks = 16384;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_energyScratch[kNoAllocMaxBlocks];

// host-side table of the array's address on each device; the array's name in
// host code is only a stand-in, so the device address has to be looked up
static double *g_scratchAddr[kNoAllocMaxDevices] = {nullptr};
static std::mutex g_scratchMu;

static double *noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    set_error("device %d outside 0..%d", device, kNoAllocMaxDevices - 1);
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_scratchMu);
  if (g_scratchAddr[device] == nullptr) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != device) {
      set_error("scratch set-up: device %d is not current", device);
      return nullptr;
    }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_energyScratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("scratch set-up on device %d failed: %s", device, cudaGetErrorString(e));
      return nullptr;
    }
    g_scratchAddr[device] = (double *)p;
  }
  return g_scratchAddr[device];
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
  sum_partials_kernel<<<1, 32, 0, c->stream>>>((int)blocks, scratch, raw);
  c->launches += 2;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("fabipb_b200_energy_noalloc: launch failed: %s", cudaGetErrorString(e));
    return 0;
  }
  return 1;
}
