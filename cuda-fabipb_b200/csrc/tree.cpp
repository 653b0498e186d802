// tree.cpp -- host construction of the panel octree and the FMM layouts.
// Compiled with -ffp-contract=off: the cell tests, box centres and the MAC
// must round exactly like the reference (which has no fused multiply-add on
// its x86-64 build) or panels can land in a different leaf.
#include "tree.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>

#include "common.cuh"

namespace fb {

// f(lo, hi) over [0, n) in contiguous chunks on the host's cores (results
// must not depend on the chunking: every caller writes disjoint outputs)
template <typename F>
static void parallel_chunks(long long n, F f) {
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 4096 || nth == 1) {
    f(0LL, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int th = 1; th < nth; th++) pool.emplace_back(f, n * th / nth, n * (th + 1) / nth);
  f(0LL, n / nth);
  for (auto &t : pool) t.join();
}

// host stage times of the tree build, printed when FABIPB_B200_TRACE is set
struct HostTimer {
  bool on = getenv("FABIPB_B200_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(const char *stage) {
    if (!on) return;
    auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "[fabipb_b200] tree.%s %.3f ms\n", stage,
            std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

bool build_octree(Octree &t, int n, const double *pts, int depth, int height, double minx,
                  double miny, double minz, double length, std::vector<int> &sorted) {
  if (depth < 1 || depth > 20 || n <= 0 || height < 0 || height > depth) {
    set_error("octree: invalid depth %d / height %d for %d points", depth, height, n);
    return false;
  }
  t = Octree();
  t.depth = depth;
  t.height = height;
  double sideLen[64];
  for (int lev = 0; lev <= depth; lev++) { sideLen[lev] = length; length *= 0.5; }

  std::vector<uint64_t> key(n);
  parallel_chunks(n, [&](long long i0, long long i1) {
    for (long long i = i0; i < i1; i++) {
      const double *x = &pts[3 * i];
      int ci = 0, cj = 0, ck = 0;
      uint64_t k = 0;
      for (int lev = 0; lev < depth; lev++) {
        int ix = (x[0] > minx + (ci + 0.5) * sideLen[lev]) ? 1 : 0;
        int iy = (x[1] > miny + (cj + 0.5) * sideLen[lev]) ? 1 : 0;
        int iz = (x[2] > minz + (ck + 0.5) * sideLen[lev]) ? 1 : 0;
        ci = 2 * ci + ix; cj = 2 * cj + iy; ck = 2 * ck + iz;
        k = (k << 3) | (uint64_t)(ix + 2 * iy + 4 * iz);
      }
      key[i] = k;
    }
  });
  // stable LSD radix sort of the item indices by their 3*depth-bit keys (the
  // order a stable comparison sort gives)
  std::vector<uint64_t> ks(key);   // keys carried along the sort
  sorted.resize(n);
  std::iota(sorted.begin(), sorted.end(), 0);
  {
    std::vector<int> tmp(n);
    std::vector<uint64_t> ktmp(n);
    const int bits = 3 * depth;
    for (int sh = 0; sh < bits; sh += 11) {
      std::vector<int> cnt(2049, 0);
      for (int i = 0; i < n; i++) cnt[((ks[i] >> sh) & 2047) + 1]++;
      for (int d = 0; d < 2048; d++) cnt[d + 1] += cnt[d];
      for (int i = 0; i < n; i++) {
        const int o = cnt[(ks[i] >> sh) & 2047]++;
        tmp[o] = sorted[i];
        ktmp[o] = ks[i];
      }
      sorted.swap(tmp);
      ks.swap(ktmp);
    }
  }

  // cubes level by level: a cube starts wherever the key prefix of the level
  // changes along the sorted items; its parent is the cube of its first item
  // one level up
  t.levStart.assign(depth + 2, 0);
  std::vector<int> prevStart;   // item starts of the previous level's cubes
  for (int lev = 0; lev <= depth; lev++) {
    const int shift = 3 * (depth - lev);
    t.levStart[lev] = t.nCubes;
    std::vector<int> starts;
    starts.reserve(lev == 0 ? 1 : prevStart.size() * 8);
    for (int i = 0; i < n; i++)
      if (i == 0 || (ks[i] >> shift) != (ks[i - 1] >> shift)) starts.push_back(i);
    const int pc0 = lev == 0 ? -1 : t.levStart[lev - 1];
    size_t p = 0;
    for (size_t q = 0; q < starts.size(); q++) {
      const int i = starts[q];
      if (lev > 0)
        while (p + 1 < prevStart.size() && prevStart[p + 1] <= i) p++;
      t.level.push_back(lev);
      t.parent.push_back(lev == 0 ? -1 : pc0 + (int)p);
      t.itemStart.push_back(i);
      t.itemCount.push_back((q + 1 < starts.size() ? starts[q + 1] : n) - i);
      t.nCubes++;
    }
    prevStart.swap(starts);
  }
  t.levStart[depth + 1] = t.nCubes;
  t.kidStart.assign(t.nCubes, -1);
  t.kidCount.assign(t.nCubes, 0);
  for (int c = 0; c < t.nCubes; c++) {
    int p = t.parent[c];
    if (p >= 0) {
      if (t.kidStart[p] < 0) t.kidStart[p] = c;
      t.kidCount[p]++;
    }
  }
  t.x.assign(3 * (size_t)t.nCubes, 0.0);
  t.lo.assign(3 * (size_t)t.nCubes, 0.0);
  t.up.assign(3 * (size_t)t.nCubes, 0.0);
  t.rad.assign(t.nCubes, 0.0);
  return true;
}

static void finish_box(Octree &t, int c) {
  const double *lo = &t.lo[3 * c], *up = &t.up[3 * c];
  t.x[3 * c] = 0.5 * (lo[0] + up[0]);
  t.x[3 * c + 1] = 0.5 * (lo[1] + up[1]);
  t.x[3 * c + 2] = 0.5 * (lo[2] + up[2]);
  double d0 = up[0] - lo[0], d1 = up[1] - lo[1], d2 = up[2] - lo[2];
  t.rad[c] = 0.5 * std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

static void parent_boxes(Octree &t) {
  for (int lev = t.depth - 1; lev >= t.height; lev--) {
    for (int c = t.levStart[lev]; c < t.levStart[lev + 1]; c++) {
      double *lo = &t.lo[3 * c], *up = &t.up[3 * c];
      int k0 = t.kidStart[c];
      for (int k = 0; k < 3; k++) { up[k] = t.up[3 * k0 + k]; lo[k] = t.lo[3 * k0 + k]; }
      for (int i = 1; i < t.kidCount[c]; i++) {
        int kid = k0 + i;
        for (int k = 0; k < 3; k++) {
          up[k] = t.up[3 * kid + k] > up[k] ? t.up[3 * kid + k] : up[k];
          lo[k] = t.lo[3 * kid + k] < lo[k] ? t.lo[3 * kid + k] : lo[k];
        }
      }
      finish_box(t, c);
    }
  }
}

void octree_boxes_panels(Octree &t, const double *vtx) {
  const int c0 = t.levStart[t.depth], c1 = t.levStart[t.depth + 1];
  parallel_chunks(c1 - c0, [&](long long a, long long b) {
  for (int c = c0 + (int)a; c < c0 + (int)b; c++) {
    double *lo = &t.lo[3 * c], *up = &t.up[3 * c];
    int p0 = t.itemStart[c];
    for (int k = 0; k < 3; k++) { up[k] = vtx[9 * (size_t)p0 + k]; lo[k] = up[k]; }
    for (int i = 0; i < t.itemCount[c]; i++) {
      for (int j = 0; j < 3; j++) {
        const double *x = &vtx[9 * (size_t)(p0 + i) + 3 * j];
        for (int k = 0; k < 3; k++) {
          up[k] = x[k] > up[k] ? x[k] : up[k];
          lo[k] = x[k] < lo[k] ? x[k] : lo[k];
        }
      }
    }
    finish_box(t, c);
  }
  });
  parent_boxes(t);
}

void octree_boxes_points(Octree &t, const double *pts, const std::vector<int> &sorted) {
  for (int c = t.levStart[t.depth]; c < t.levStart[t.depth + 1]; c++) {
    double *lo = &t.lo[3 * c], *up = &t.up[3 * c];
    int s0 = t.itemStart[c];
    for (int k = 0; k < 3; k++) { up[k] = lo[k] = pts[3 * (size_t)sorted[s0] + k]; }
    for (int i = 1; i < t.itemCount[c]; i++) {
      const double *x = &pts[3 * (size_t)sorted[s0 + i]];
      for (int k = 0; k < 3; k++) {
        up[k] = x[k] > up[k] ? x[k] : up[k];
        lo[k] = x[k] < lo[k] ? x[k] : lo[k];
      }
    }
    finish_box(t, c);
  }
  parent_boxes(t);
}

static int mac_near(const Octree &t, int c1, int c2, double eta0) {
  if (c1 == c2) return 2;
  double d0 = t.x[3 * c1] - t.x[3 * c2];
  double d1 = t.x[3 * c1 + 1] - t.x[3 * c2 + 1];
  double d2 = t.x[3 * c1 + 2] - t.x[3 * c2 + 2];
  double dist = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (dist < 1e-15) return 1;
  double eta = (t.rad[c1] + t.rad[c2]) / dist;
  return (eta < eta0) ? 0 : 1;
}

void octree_neighbours(Octree &t, double eta0) {
  t.nbrStart.assign(t.nCubes, -1);
  t.nNbr1.assign(t.nCubes, 0);
  t.nNbr2.assign(t.nCubes, 0);
  t.nbr.clear();
  // level by level (a cube's candidates are the children of its parent's near
  // list): the cubes of a level in parallel into their own lists, then
  // appended in cube order
  for (int lev = t.height; lev <= t.depth; lev++) {
    const int c0 = t.levStart[lev], nc = t.levStart[lev + 1] - c0;
    std::vector<std::vector<int>> lists(nc);
    std::vector<int> n1(nc), n2(nc);
    parallel_chunks(nc, [&](long long a, long long b) {
      std::vector<int> cands;
      for (int ci = (int)a; ci < (int)b; ci++) {
        const int c = c0 + ci;
        cands.clear();
        if (lev == t.height) {
          for (int d = t.levStart[lev]; d < t.levStart[lev + 1]; d++) cands.push_back(d);
        } else {
          int p = t.parent[c];
          for (int q = 0; q < t.nNbr1[p]; q++) {
            int np = t.nbr[t.nbrStart[p] + q];
            for (int k = 0; k < t.kidCount[np]; k++) cands.push_back(t.kidStart[np] + k);
          }
        }
        int nNear = 0;
        for (int d : cands) if (mac_near(t, c, d, eta0)) nNear++;
        std::vector<int> &out = lists[ci];
        out.assign(cands.size(), 0);
        int i1 = 1, i2 = nNear;
        for (int d : cands) {
          int f = mac_near(t, c, d, eta0);
          if (f == 1) out[i1++] = d;
          else if (f == 2) out[0] = d;
          else out[i2++] = d;
        }
        n1[ci] = i1;
        n2[ci] = i2;
      }
    });
    size_t total = t.nbr.size();
    for (int ci = 0; ci < nc; ci++) total += lists[ci].size();
    t.nbr.reserve(total);
    for (int ci = 0; ci < nc; ci++) {
      t.nbrStart[c0 + ci] = (int)t.nbr.size();
      t.nNbr1[c0 + ci] = n1[ci];
      t.nNbr2[c0 + ci] = n2[ci];
      t.nbr.insert(t.nbr.end(), lists[ci].begin(), lists[ci].end());
    }
  }
}

bool build_panel_tree(PanelTree &pt, int n, const double *vtx, int depth, int height,
                      double sep_ratio, int order, int order_mom) {
  // loopPanels (gkSetup.c:90-128): vertex extents and centroids in input order
  // (extents: min/max per chunk, then over the chunks -- the same values in any order)
  double minx = vtx[0], maxx = vtx[0], miny = vtx[1], maxy = vtx[1], minz = vtx[2], maxz = vtx[2];
  std::vector<double> ctr(3 * (size_t)n);
  std::mutex mu;
  parallel_chunks(n, [&](long long i0, long long i1) {
    double lx = vtx[0], ux = vtx[0], ly = vtx[1], uy = vtx[1], lz = vtx[2], uz = vtx[2];
    for (long long i = i0; i < i1; i++) {
      const double *v = &vtx[9 * (size_t)i];
      for (int k = 0; k < 3; k++) {
        const double *x = &v[3 * k];
        ux = x[0] > ux ? x[0] : ux; lx = lx > x[0] ? x[0] : lx;
        uy = x[1] > uy ? x[1] : uy; ly = ly > x[1] ? x[1] : ly;
        uz = x[2] > uz ? x[2] : uz; lz = lz > x[2] ? x[2] : lz;
      }
      for (int k = 0; k < 3; k++) ctr[3 * (size_t)i + k] = kOneThird * (v[k] + v[3 + k] + v[6 + k]);
    }
    std::lock_guard<std::mutex> lk(mu);
    maxx = ux > maxx ? ux : maxx; minx = minx > lx ? lx : minx;
    maxy = uy > maxy ? uy : maxy; miny = miny > ly ? ly : miny;
    maxz = uz > maxz ? uz : maxz; minz = minz > lz ? lz : minz;
  });
  HostTimer ht;
  double length = (maxx - minx) > (maxy - miny) ? (maxx - minx) : (maxy - miny);
  length = (maxz - minz) > length ? (maxz - minz) : length;
  pt.n = n;
  if (!build_octree(pt.t, n, ctr.data(), depth, height, minx, miny, minz, length, pt.order))
    return false;
  ht.mark("cells_and_sort");
  std::vector<double> vt(9 * (size_t)n);
  parallel_chunks(n, [&](long long i0, long long i1) {
    for (long long i = i0; i < i1; i++) memcpy(&vt[9 * i], &vtx[9 * (size_t)pt.order[i]], 9 * sizeof(double));
  });
  octree_boxes_panels(pt.t, vt.data());
  ht.mark("boxes");
  octree_neighbours(pt.t, sep_ratio);
  ht.mark("neighbours");
  if (!finish_panel_tree(pt, order, order_mom)) return false;
  ht.mark("layouts");
  return true;
}

bool finish_panel_tree(PanelTree &pt, int order, int order_mom) {
  Octree &t = pt.t;
  const int depth = t.depth, height = t.height;

  // getOrders (gkSetup.c:42-81)
  pt.ordMom.assign(depth + 1, 0);
  pt.ordM2L.assign(depth + 1, 0);
  if (order > 0) {
    for (int l = 0; l <= depth; l++) pt.ordM2L[l] = pt.ordMom[l] = order;
    pt.maxOrder = order;
  } else {
    pt.ordM2L[depth] = -order;
    for (int l = depth - 1; l >= height; l--) pt.ordM2L[l] = pt.ordM2L[l + 1] + 1;
    pt.maxOrder = pt.ordM2L[height];
    for (int l = depth; l >= height; l--)
      pt.ordMom[l] = order_mom >= 0 ? std::min(pt.ordM2L[l] + order_mom, pt.maxOrder) : pt.maxOrder;
  }
  if (pt.maxOrder > kMaxOrder) {
    set_error("expansion order %d exceeds the device limit %d", pt.maxOrder, kMaxOrder);
    return false;
  }

  // buildApplyLayout (fmm.c:234-268): near pairs by destination leaf, self first
  pt.nLeaves = t.levStart[depth + 1] - t.levStart[depth];
  pt.leafStart.resize(pt.nLeaves);
  pt.leafCount.resize(pt.nLeaves);
  pt.leafCube.resize(pt.nLeaves);
  pt.nearOff.assign(pt.nLeaves + 1, 0);
  pt.nearSrc.clear();
  pt.nearDst.clear();
  {
    size_t tot = 0;
    for (int L = 0; L < pt.nLeaves; L++) tot += t.nNbr1[t.levStart[depth] + L];
    pt.nearSrc.reserve(tot);
    pt.nearDst.reserve(tot);
  }
  for (int L = 0; L < pt.nLeaves; L++) {
    int c = t.levStart[depth] + L;
    pt.leafCube[L] = c;
    pt.leafStart[L] = t.itemStart[c];
    pt.leafCount[L] = t.itemCount[c];
    pt.nearOff[L] = (int)pt.nearSrc.size();
    for (int k = 0; k < t.nNbr1[c]; k++) {
      pt.nearSrc.push_back(t.nbr[t.nbrStart[c] + k] - t.levStart[depth]);
      pt.nearDst.push_back(L);
    }
  }
  pt.nearOff[pt.nLeaves] = (int)pt.nearSrc.size();

  // buildFmmCubeLayout (fmm.c:295-324): levels depth..height
  pt.cubeFmm.assign(t.nCubes, -1);
  pt.fmmCube.clear();
  pt.fmmLevelStart.assign(depth + 1, 0);
  pt.fmmLevelCount.assign(depth + 1, 0);
  for (int lev = depth; lev >= height; lev--) {
    pt.fmmLevelStart[lev] = (int)pt.fmmCube.size();
    for (int c = t.levStart[lev]; c < t.levStart[lev + 1]; c++) {
      pt.cubeFmm[c] = (int)pt.fmmCube.size();
      pt.fmmCube.push_back(c);
    }
    pt.fmmLevelCount[lev] = (int)pt.fmmCube.size() - pt.fmmLevelStart[lev];
  }
  pt.nFmm = (int)pt.fmmCube.size();

  // buildM2LPairList (fmm.c:326-373): interaction list in reverse order
  pt.m2lOff.assign(pt.nFmm + 1, 0);
  pt.m2lSrc.clear();
  pt.m2lPairSrc.clear();
  pt.m2lPairDst.clear();
  {
    size_t tot = 0;
    for (int f = 0; f < pt.nFmm; f++) tot += t.nNbr2[pt.fmmCube[f]] - t.nNbr1[pt.fmmCube[f]];
    pt.m2lSrc.reserve(tot);
    pt.m2lPairSrc.reserve(tot);
    pt.m2lPairDst.reserve(tot);
  }
  for (int f = 0; f < pt.nFmm; f++) {
    int c = pt.fmmCube[f];
    pt.m2lOff[f] = (int)pt.m2lSrc.size();
    for (int i = t.nNbr2[c] - 1; i >= t.nNbr1[c]; i--) {
      int s = pt.cubeFmm[t.nbr[t.nbrStart[c] + i]];
      pt.m2lSrc.push_back(s);
      pt.m2lPairSrc.push_back(s);
      pt.m2lPairDst.push_back(f);
    }
  }
  pt.m2lOff[pt.nFmm] = (int)pt.m2lSrc.size();
  return true;
}

}  // namespace fb
