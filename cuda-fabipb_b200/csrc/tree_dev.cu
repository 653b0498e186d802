// tree_dev.cu -- the panel octree built on the device.
//
// Produces exactly the PanelTree of build_panel_tree (tree.cpp), which
// reproduces the reference's loopPanels / goDown / linkcubes / getEnclBoxs /
// getNbrs (src/gkSetup.c:90-437):
//   extents, centroids  one pass over the panels; block min/max partials
//   cell keys           per panel, goDown's strict '>' tests level by level
//                       against min + (i + 0.5) sideLen[level]
//   panel order         stable radix sort (cub) of the 3*depth-bit keys: the
//                       depth-first order with children in index order, and
//                       input order inside a leaf
//   cubes per level     where the level's key prefix changes along the sorted
//                       panels (an exclusive scan of the change flags); a
//                       cube's parent is the previous level's cube of its
//                       first panel
//   boxes               leaf boxes from the panels' vertices, parents from
//                       their children bottom-up to the top FMM level; centre
//                       and radius of the vertex bounding box
//   near lists          level by level from the top FMM level, candidates the
//                       children of the parent's near cubes; self first, then
//                       the cubes that fail the MAC (near), then those that pass
//                       (interaction list), each group in candidate order
// Every product, sum, square root and quotient of the geometry is rounded
// separately (no fused multiply-add), as the reference's x86-64 build and the
// host builder (compiled with -ffp-contract=off) compute them, so every panel
// lands in the same leaf and every MAC decision is the same.  The cube records
// are copied back to the host, where finish_panel_tree builds the flattened
// layouts; the panels are gathered into tree order on the device.
#include <cfloat>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "context.cuh"

namespace fb {

constexpr int kTreeThreads = 256;
constexpr int kTreeExtentBlocks = 4 * 148;

struct TreeSides {
  double len[21];
};

// centroid (loopPanels: (v0 + v1 + v2) / 3 as kOneThird * sum) of every panel
// and the block's vertex extents part[6 * block] = (min xyz, max xyz)
__global__ void __launch_bounds__(kTreeThreads)
tree_extent_kernel(int n, const double *__restrict__ vtx, double *ctr, double *part) {
  __shared__ double red[6][kTreeThreads];
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, up[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double *v = vtx + 9 * (size_t)i;
    for (int k = 0; k < 3; k++)
      for (int d = 0; d < 3; d++) {
        const double x = v[3 * k + d];
        up[d] = x > up[d] ? x : up[d];
        lo[d] = lo[d] > x ? x : lo[d];
      }
    for (int d = 0; d < 3; d++) ctr[3 * (size_t)i + d] = __dmul_rn(kOneThird, __dadd_rn(__dadd_rn(v[d], v[3 + d]), v[6 + d]));
  }
  for (int d = 0; d < 3; d++) {
    red[d][threadIdx.x] = lo[d];
    red[3 + d][threadIdx.x] = up[d];
  }
  __syncthreads();
  for (int m = kTreeThreads / 2; m > 0; m >>= 1) {
    if ((int)threadIdx.x < m)
      for (int d = 0; d < 3; d++) {
        const double a = red[d][threadIdx.x + m], b = red[3 + d][threadIdx.x + m];
        red[d][threadIdx.x] = red[d][threadIdx.x] > a ? a : red[d][threadIdx.x];
        red[3 + d][threadIdx.x] = b > red[3 + d][threadIdx.x] ? b : red[3 + d][threadIdx.x];
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) part[6 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

// goDown's cell of every centroid, as a 3*depth-bit key with the 3-bit digit
// ix + 2 iy + 4 iz per level (src/gkSetup.c:142-183)
__global__ void tree_keys_kernel(int n, const double *__restrict__ ctr, double minx, double miny, double minz,
                                 TreeSides sl, int depth, unsigned long long *key, int *idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = ctr[3 * (size_t)i], y = ctr[3 * (size_t)i + 1], z = ctr[3 * (size_t)i + 2];
  int ci = 0, cj = 0, ck = 0;
  unsigned long long k = 0;
  for (int lev = 0; lev < depth; lev++) {
    const int ix = x > __dadd_rn(minx, __dmul_rn((double)ci + 0.5, sl.len[lev])) ? 1 : 0;
    const int iy = y > __dadd_rn(miny, __dmul_rn((double)cj + 0.5, sl.len[lev])) ? 1 : 0;
    const int iz = z > __dadd_rn(minz, __dmul_rn((double)ck + 0.5, sl.len[lev])) ? 1 : 0;
    ci = 2 * ci + ix;
    cj = 2 * cj + iy;
    ck = 2 * ck + iz;
    k = (k << 3) | (unsigned long long)(ix + 2 * iy + 4 * iz);
  }
  key[i] = k;
  idx[i] = i;
}

// flag[i] = 1 where the level's key prefix (key >> shift) starts a new cube
__global__ void tree_level_flags_kernel(int n, const unsigned long long *__restrict__ key, int shift, int *flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = (i == 0 || (key[i] >> shift) != (key[i - 1] >> shift)) ? 1 : 0;
}

// the level's cubes: first panel, parent (the previous level's cube of that
// panel), and every panel's cube index within the level
__global__ void tree_level_emit_kernel(int n, const int *__restrict__ flag, const int *__restrict__ pos,
                                       const int *__restrict__ prevCube, int prevLevStart, int *start, int *parent,
                                       int *cubeOfItem) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flag[i]) {
    start[pos[i]] = i;
    parent[pos[i]] = prevCube ? prevLevStart + prevCube[i] : -1;
  }
  cubeOfItem[i] = pos[i] + flag[i] - 1;
}

// panels into tree order
__global__ void tree_gather_kernel(int n, const int *__restrict__ order, const double *__restrict__ vtxIn,
                                   const double *__restrict__ nrmIn, const double *__restrict__ areaIn, double *vtx,
                                   double *nrm, double *area) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = order[i];
  for (int k = 0; k < 9; k++) vtx[9 * (size_t)i + k] = vtxIn[9 * (size_t)o + k];
  for (int k = 0; k < 3; k++) nrm[3 * (size_t)i + k] = nrmIn[3 * (size_t)o + k];
  area[i] = areaIn[o];
}

// centre and radius of a cube's box (finish_box in tree.cpp)
__device__ __forceinline__ void tree_finish_box(const double *lo, const double *up, double *x, double *rad) {
  for (int k = 0; k < 3; k++) x[k] = __dmul_rn(0.5, __dadd_rn(lo[k], up[k]));
  const double d0 = __dsub_rn(up[0], lo[0]), d1 = __dsub_rn(up[1], lo[1]), d2 = __dsub_rn(up[2], lo[2]);
  *rad = __dmul_rn(0.5, __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2))));
}

// leaf boxes: the extents of the leaf panels' vertices (getEnclBoxs)
__global__ void tree_leaf_box_kernel(int c0, int nc, const int *__restrict__ itemStart,
                                     const int *__restrict__ itemCount, const double *__restrict__ vtx, double *lo,
                                     double *up, double *x, double *rad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc) return;
  const int c = c0 + t;
  const int p0 = itemStart[c], cnt = itemCount[c];
  double l[3], u[3];
  for (int k = 0; k < 3; k++) u[k] = l[k] = vtx[9 * (size_t)p0 + k];
  for (int i = 0; i < cnt; i++)
    for (int j = 0; j < 3; j++) {
      const double *v = vtx + 9 * (size_t)(p0 + i) + 3 * j;
      for (int k = 0; k < 3; k++) {
        u[k] = v[k] > u[k] ? v[k] : u[k];
        l[k] = v[k] < l[k] ? v[k] : l[k];
      }
    }
  for (int k = 0; k < 3; k++) {
    lo[3 * (size_t)c + k] = l[k];
    up[3 * (size_t)c + k] = u[k];
  }
  tree_finish_box(l, u, x + 3 * (size_t)c, rad + c);
}

// a level's boxes from its children's (parent_boxes in tree.cpp)
__global__ void tree_parent_box_kernel(int c0, int nc, const int *__restrict__ kidStart,
                                       const int *__restrict__ kidCount, double *lo, double *up, double *x,
                                       double *rad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc) return;
  const int c = c0 + t, k0 = kidStart[c];
  double l[3], u[3];
  for (int k = 0; k < 3; k++) {
    u[k] = up[3 * (size_t)k0 + k];
    l[k] = lo[3 * (size_t)k0 + k];
  }
  for (int i = 1; i < kidCount[c]; i++)
    for (int k = 0; k < 3; k++) {
      const double a = up[3 * (size_t)(k0 + i) + k], b = lo[3 * (size_t)(k0 + i) + k];
      u[k] = a > u[k] ? a : u[k];
      l[k] = b < l[k] ? b : l[k];
    }
  for (int k = 0; k < 3; k++) {
    lo[3 * (size_t)c + k] = l[k];
    up[3 * (size_t)c + k] = u[k];
  }
  tree_finish_box(l, u, x + 3 * (size_t)c, rad + c);
}

// the reference's MAC (src/gkSetup.c:332-349): 2 self, 1 near, 0 far
__device__ __forceinline__ int tree_mac(const double *__restrict__ x, const double *__restrict__ rad, int c1, int c2,
                                        double eta0) {
  if (c1 == c2) return 2;
  const double d0 = __dsub_rn(x[3 * (size_t)c1], x[3 * (size_t)c2]);
  const double d1 = __dsub_rn(x[3 * (size_t)c1 + 1], x[3 * (size_t)c2 + 1]);
  const double d2 = __dsub_rn(x[3 * (size_t)c1 + 2], x[3 * (size_t)c2 + 2]);
  const double dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
  if (dist < 1e-15) return 1;
  const double eta = __ddiv_rn(__dadd_rn(rad[c1], rad[c2]), dist);
  return (eta < eta0) ? 0 : 1;
}

// candidate cube q of cube c: at the top FMM level every cube of the level,
// below it the children of the parent's near cubes (nbrP: the parent level's
// lists, relative offsets)
struct TreeCands {
  int top;                 // 1 at the top FMM level
  int lev0, levN;          // the level's first cube and cube count
  const int *parent, *kidStart, *kidCount;
  const int *nbrStartP, *nNbr1P, *nbrP;   // parent level (nbrStartP indexed by cube id)
};

__device__ __forceinline__ int tree_cand_count(const TreeCands &C, int c) {
  if (C.top) return C.levN;
  const int p = C.parent[c];
  int s = 0;
  for (int q = 0; q < C.nNbr1P[p]; q++) s += C.kidCount[C.nbrP[C.nbrStartP[p] + q]];
  return s;
}

template <typename F>
__device__ __forceinline__ void tree_cand_each(const TreeCands &C, int c, F f) {
  if (C.top) {
    for (int d = C.lev0; d < C.lev0 + C.levN; d++) f(d);
    return;
  }
  const int p = C.parent[c];
  for (int q = 0; q < C.nNbr1P[p]; q++) {
    const int np = C.nbrP[C.nbrStartP[p] + q];
    for (int k = 0; k < C.kidCount[np]; k++) f(C.kidStart[np] + k);
  }
}

__global__ void tree_nbr_count_kernel(TreeCands C, int *count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C.levN) return;
  count[t] = tree_cand_count(C, C.lev0 + t);
}

// a cube's list at off[t]: self, near cubes, interaction cubes
__global__ void tree_nbr_fill_kernel(TreeCands C, const double *__restrict__ x, const double *__restrict__ rad,
                                     double eta0, const int *__restrict__ off, int *nbr, int *nbrStart, int *nNbr1,
                                     int *nNbr2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C.levN) return;
  const int c = C.lev0 + t;
  int nNear = 0;
  tree_cand_each(C, c, [&](int d) { nNear += tree_mac(x, rad, c, d, eta0) ? 1 : 0; });
  int *out = nbr + off[t];
  int i1 = 1, i2 = nNear;
  tree_cand_each(C, c, [&](int d) {
    const int f = tree_mac(x, rad, c, d, eta0);
    if (f == 1) out[i1++] = d;
    else if (f == 2) out[0] = d;
    else out[i2++] = d;
  });
  nbrStart[c] = off[t];
  nNbr1[c] = i1;
  nNbr2[c] = i2;
}

// releases a scratch arena on every return path
struct ArenaScope {
  DevArena &a;
  ~ArenaScope() { a.release(); }
};

template <typename T>
static bool d2h_vec(std::vector<T> &h, const T *d, size_t n, cudaStream_t s) {
  h.resize(n);
  if (n) FB_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  return true;
}

// The panel tree of the input panels (vtx, nrm, area on the host, input
// order), built on the device into c.pt; the panels in tree order are left in
// c.d_vtx, c.d_nrm, c.d_area.
bool build_panel_tree_device(Context &c, const double *vtxIn, const double *nrmIn, const double *areaIn) {
  const int n = c.n, depth = c.prm.depth, height = c.prm.height;
  FB_CHECK(depth >= 1 && depth <= 20 && height >= 0 && height <= depth && n > 0,
           "octree: invalid depth %d / height %d for %d panels", depth, height, n);
  cudaStream_t s = c.stream;
  PanelTree &pt = c.pt;
  pt = PanelTree();
  pt.n = n;
  Octree &t = pt.t;
  t.depth = depth;
  t.height = height;
  DevArena tmp;
  ArenaScope tmpScope{tmp};
  double *d_vin = nullptr, *d_nin = nullptr, *d_ain = nullptr, *d_ctr = nullptr, *d_part = nullptr;
  unsigned long long *d_key = nullptr, *d_keyS = nullptr;
  int *d_idx = nullptr, *d_order = nullptr, *d_flag = nullptr, *d_pos = nullptr, *d_cubeA = nullptr,
      *d_cubeB = nullptr;
  if (!tmp.alloc_n(&d_vin, 9 * (size_t)n) || !tmp.alloc_n(&d_nin, 3 * (size_t)n) || !tmp.alloc_n(&d_ain, (size_t)n) ||
      !tmp.alloc_n(&d_ctr, 3 * (size_t)n) || !tmp.alloc_n(&d_part, 6 * (size_t)kTreeExtentBlocks) ||
      !tmp.alloc_n(&d_key, (size_t)n) || !tmp.alloc_n(&d_keyS, (size_t)n) || !tmp.alloc_n(&d_idx, (size_t)n) ||
      !tmp.alloc_n(&d_flag, (size_t)n) || !tmp.alloc_n(&d_pos, (size_t)n) || !tmp.alloc_n(&d_cubeA, (size_t)n) ||
      !tmp.alloc_n(&d_cubeB, (size_t)n) || !tmp.alloc_n(&d_order, (size_t)n) ||
      !c.arena.alloc_n(&c.d_vtx, 9 * (size_t)n) || !c.arena.alloc_n(&c.d_nrm, 3 * (size_t)n) ||
      !c.arena.alloc_n(&c.d_area, (size_t)n))
    return false;
  FB_CUDA(cudaMemcpyAsync(d_vin, vtxIn, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  FB_CUDA(cudaMemcpyAsync(d_nin, nrmIn, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  FB_CUDA(cudaMemcpyAsync(d_ain, areaIn, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));

  // extents and centroids
  tree_extent_kernel<<<kTreeExtentBlocks, kTreeThreads, 0, s>>>(n, d_vin, d_ctr, d_part);
  c.launches += 1;
  std::vector<double> part;
  if (!d2h_vec(part, d_part, 6 * (size_t)kTreeExtentBlocks, s)) return false;
  FB_CUDA(cudaStreamSynchronize(s));
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, up[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int b = 0; b < kTreeExtentBlocks; b++)
    for (int d = 0; d < 3; d++) {
      lo[d] = lo[d] > part[6 * b + d] ? part[6 * b + d] : lo[d];
      up[d] = part[6 * b + 3 + d] > up[d] ? part[6 * b + 3 + d] : up[d];
    }
  double length = (up[0] - lo[0]) > (up[1] - lo[1]) ? (up[0] - lo[0]) : (up[1] - lo[1]);
  length = (up[2] - lo[2]) > length ? (up[2] - lo[2]) : length;
  TreeSides sl{};
  for (int lev = 0; lev <= depth; lev++) {
    sl.len[lev] = length;
    length *= 0.5;
  }

  // keys and the stable sort
  tree_keys_kernel<<<ceil_div(n, kTreeThreads), kTreeThreads, 0, s>>>(n, d_ctr, lo[0], lo[1], lo[2], sl, depth,
                                                                      d_key, d_idx);
  c.launches += 1;
  size_t tb = 0, tb2 = 0;
  FB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_key, d_keyS, d_idx, d_order, n, 0, 3 * depth, s));
  FB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, d_flag, d_pos, n, s));
  void *d_tmp = nullptr;
  if (!tmp.alloc(&d_tmp, std::max(tb, tb2))) return false;
  FB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tb, d_key, d_keyS, d_idx, d_order, n, 0, 3 * depth, s));
  c.launches += 4;

  // cubes level by level
  t.levStart.assign(depth + 2, 0);
  int *prev = nullptr, *cur = d_cubeA;
  std::vector<int> cnt2(2);
  int *d_start = nullptr, *d_parent = nullptr;
  if (!tmp.alloc_n(&d_start, (size_t)n) || !tmp.alloc_n(&d_parent, (size_t)n)) return false;
  for (int lev = 0; lev <= depth; lev++) {
    const int shift = 3 * (depth - lev);
    tree_level_flags_kernel<<<ceil_div(n, kTreeThreads), kTreeThreads, 0, s>>>(n, d_keyS, shift, d_flag);
    FB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tb2, d_flag, d_pos, n, s));
    tree_level_emit_kernel<<<ceil_div(n, kTreeThreads), kTreeThreads, 0, s>>>(
        n, d_flag, d_pos, prev, lev == 0 ? 0 : t.levStart[lev - 1], d_start, d_parent, cur);
    c.launches += 3;
    FB_CUDA(cudaMemcpyAsync(&cnt2[0], d_pos + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(&cnt2[1], d_flag + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    const int nc = cnt2[0] + cnt2[1];
    t.levStart[lev] = t.nCubes;
    const size_t base = t.itemStart.size();
    t.itemStart.resize(base + nc);
    t.parent.resize(base + nc);
    FB_CUDA(cudaMemcpyAsync(t.itemStart.data() + base, d_start, nc * sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(t.parent.data() + base, d_parent, nc * sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nc; q++) {
      t.level.push_back(lev);
      t.itemCount.push_back((q + 1 < nc ? t.itemStart[base + q + 1] : n) - t.itemStart[base + q]);
    }
    t.nCubes += nc;
    prev = cur;
    cur = (cur == d_cubeA) ? d_cubeB : d_cubeA;
  }
  t.levStart[depth + 1] = t.nCubes;
  t.kidStart.assign(t.nCubes, -1);
  t.kidCount.assign(t.nCubes, 0);
  for (int cc = 0; cc < t.nCubes; cc++) {
    const int p = t.parent[cc];
    if (p >= 0) {
      if (t.kidStart[p] < 0) t.kidStart[p] = cc;
      t.kidCount[p]++;
    }
  }
  if (!d2h_vec(pt.order, d_order, (size_t)n, s)) return false;

  // panels in tree order; boxes
  tree_gather_kernel<<<ceil_div(n, kTreeThreads), kTreeThreads, 0, s>>>(n, d_order, d_vin, d_nin, d_ain, c.d_vtx,
                                                                         c.d_nrm, c.d_area);
  c.launches += 1;
  const int nCubes = t.nCubes;
  int *d_itemStart = nullptr, *d_itemCount = nullptr, *d_kidStart = nullptr, *d_kidCount = nullptr,
      *d_parentAll = nullptr;
  double *d_lo = nullptr, *d_up = nullptr, *d_x = nullptr, *d_rad = nullptr;
  if (!tmp.upload(&d_itemStart, t.itemStart, s) || !tmp.upload(&d_itemCount, t.itemCount, s) ||
      !tmp.upload(&d_kidStart, t.kidStart, s) || !tmp.upload(&d_kidCount, t.kidCount, s) ||
      !tmp.upload(&d_parentAll, t.parent, s) || !tmp.alloc_n(&d_lo, 3 * (size_t)nCubes) ||
      !tmp.alloc_n(&d_up, 3 * (size_t)nCubes) || !tmp.alloc_n(&d_x, 3 * (size_t)nCubes) ||
      !tmp.alloc_n(&d_rad, (size_t)nCubes))
    return false;
  FB_CUDA(cudaMemsetAsync(d_lo, 0, 3 * (size_t)nCubes * sizeof(double), s));
  FB_CUDA(cudaMemsetAsync(d_up, 0, 3 * (size_t)nCubes * sizeof(double), s));
  FB_CUDA(cudaMemsetAsync(d_x, 0, 3 * (size_t)nCubes * sizeof(double), s));
  FB_CUDA(cudaMemsetAsync(d_rad, 0, (size_t)nCubes * sizeof(double), s));
  {
    const int c0 = t.levStart[depth], nc = t.levStart[depth + 1] - c0;
    tree_leaf_box_kernel<<<ceil_div(nc, 128), 128, 0, s>>>(c0, nc, d_itemStart, d_itemCount, c.d_vtx, d_lo, d_up,
                                                           d_x, d_rad);
    c.launches += 1;
  }
  for (int lev = depth - 1; lev >= height; lev--) {
    const int c0 = t.levStart[lev], nc = t.levStart[lev + 1] - c0;
    tree_parent_box_kernel<<<ceil_div(nc, 128), 128, 0, s>>>(c0, nc, d_kidStart, d_kidCount, d_lo, d_up, d_x, d_rad);
    c.launches += 1;
  }
  FB_CUDA(cudaGetLastError());

  // near / interaction lists level by level
  t.nbrStart.assign(nCubes, -1);
  t.nNbr1.assign(nCubes, 0);
  t.nNbr2.assign(nCubes, 0);
  t.nbr.clear();
  int *d_nbrStart = nullptr, *d_nNbr1 = nullptr, *d_nNbr2 = nullptr, *d_count = nullptr, *d_off = nullptr;
  if (!tmp.alloc_n(&d_nbrStart, (size_t)nCubes) || !tmp.alloc_n(&d_nNbr1, (size_t)nCubes) ||
      !tmp.alloc_n(&d_nNbr2, (size_t)nCubes) || !tmp.alloc_n(&d_count, (size_t)nCubes + 1) ||
      !tmp.alloc_n(&d_off, (size_t)nCubes + 1))
    return false;
  int *d_nbrPrev = nullptr;
  for (int lev = height; lev <= depth; lev++) {
    const int c0 = t.levStart[lev], nc = t.levStart[lev + 1] - c0;
    TreeCands C{lev == height ? 1 : 0, c0, nc, d_parentAll, d_kidStart, d_kidCount, d_nbrStart, d_nNbr1, d_nbrPrev};
    tree_nbr_count_kernel<<<ceil_div(nc, 128), 128, 0, s>>>(C, d_count);
    FB_CUDA(cudaMemsetAsync(d_count + nc, 0, sizeof(int), s));
    size_t tb3 = 0;
    FB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb3, d_count, d_off, nc + 1, s));
    void *d_tmp3 = nullptr;
    DevArena lvl;
    ArenaScope lvlScope{lvl};
    if (!lvl.alloc(&d_tmp3, tb3)) return false;
    FB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp3, tb3, d_count, d_off, nc + 1, s));
    int total = 0;
    FB_CUDA(cudaMemcpyAsync(&total, d_off + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    int *d_nbrLev = nullptr;
    if (!tmp.alloc_n(&d_nbrLev, (size_t)std::max(total, 1))) return false;
    tree_nbr_fill_kernel<<<ceil_div(nc, 128), 128, 0, s>>>(C, d_x, d_rad, c.prm.sep_ratio, d_off, d_nbrLev,
                                                           d_nbrStart, d_nNbr1, d_nNbr2);
    c.launches += 3;
    FB_CUDA(cudaGetLastError());
    const size_t base = t.nbr.size();
    t.nbr.resize(base + total);
    std::vector<int> st(nc);
    FB_CUDA(cudaMemcpyAsync(t.nbr.data() + base, d_nbrLev, (size_t)total * sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(st.data(), d_nbrStart + c0, (size_t)nc * sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(t.nNbr1.data() + c0, d_nNbr1 + c0, (size_t)nc * sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(t.nNbr2.data() + c0, d_nNbr2 + c0, (size_t)nc * sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nc; q++) t.nbrStart[c0 + q] = (int)base + st[q];
    d_nbrPrev = d_nbrLev;   // the next level's candidates read this level's lists (relative offsets)
  }
  if (!d2h_vec(t.x, d_x, 3 * (size_t)nCubes, s) || !d2h_vec(t.rad, d_rad, (size_t)nCubes, s) ||
      !d2h_vec(t.lo, d_lo, 3 * (size_t)nCubes, s) || !d2h_vec(t.up, d_up, 3 * (size_t)nCubes, s))
    return false;
  FB_CUDA(cudaStreamSynchronize(s));
  return finish_panel_tree(pt, c.prm.order, c.prm.order_mom);
}

}  // namespace fb
