// tree.cpp -- host construction of the panel octree and the FMM layouts.
// Compiled with -ffp-contract=off: the cell tests, box centres and the MAC
// must round exactly like the reference (which has no fused multiply-add on
// its x86-64 build) or panels can land in a different leaf.
#include "tree.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "common.cuh"

namespace fb {

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
  for (int i = 0; i < n; i++) {
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
  sorted.resize(n);
  std::iota(sorted.begin(), sorted.end(), 0);
  std::stable_sort(sorted.begin(), sorted.end(), [&](int a, int b) { return key[a] < key[b]; });

  t.levStart.assign(depth + 2, 0);
  std::vector<int> cubeOf(n), cubeOfPrev(n, -1);
  for (int lev = 0; lev <= depth; lev++) {
    int shift = 3 * (depth - lev);
    uint64_t cur = 0;
    t.levStart[lev] = t.nCubes;
    for (int i = 0; i < n; i++) {
      uint64_t pref = key[sorted[i]] >> shift;
      if (i == 0 || pref != cur) {
        t.level.push_back(lev);
        t.parent.push_back(lev == 0 ? -1 : cubeOfPrev[i]);
        t.itemStart.push_back(i);
        t.itemCount.push_back(0);
        t.nCubes++;
        cur = pref;
      }
      t.itemCount[t.nCubes - 1]++;
      cubeOf[i] = t.nCubes - 1;
    }
    cubeOfPrev.swap(cubeOf);
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
  for (int c = t.levStart[t.depth]; c < t.levStart[t.depth + 1]; c++) {
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
  std::vector<int> cands;
  for (int lev = t.height; lev <= t.depth; lev++) {
    for (int c = t.levStart[lev]; c < t.levStart[lev + 1]; c++) {
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
      size_t base = t.nbr.size();
      t.nbr.resize(base + cands.size());
      int i1 = 1, i2 = nNear;
      for (int d : cands) {
        int f = mac_near(t, c, d, eta0);
        if (f == 1) t.nbr[base + i1++] = d;
        else if (f == 2) t.nbr[base] = d;
        else t.nbr[base + i2++] = d;
      }
      t.nbrStart[c] = (int)base;
      t.nNbr1[c] = i1;
      t.nNbr2[c] = i2;
    }
  }
}

bool build_panel_tree(PanelTree &pt, int n, const double *vtx, int depth, int height,
                      double sep_ratio, int order, int order_mom) {
  // loopPanels (gkSetup.c:90-128): vertex extents and centroids in input order
  double minx = vtx[0], maxx = vtx[0], miny = vtx[1], maxy = vtx[1], minz = vtx[2], maxz = vtx[2];
  std::vector<double> ctr(3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    const double *v = &vtx[9 * (size_t)i];
    for (int k = 0; k < 3; k++) {
      const double *x = &v[3 * k];
      maxx = x[0] > maxx ? x[0] : maxx; minx = minx > x[0] ? x[0] : minx;
      maxy = x[1] > maxy ? x[1] : maxy; miny = miny > x[1] ? x[1] : miny;
      maxz = x[2] > maxz ? x[2] : maxz; minz = minz > x[2] ? x[2] : minz;
    }
    for (int k = 0; k < 3; k++) ctr[3 * (size_t)i + k] = kOneThird * (v[k] + v[3 + k] + v[6 + k]);
  }
  double length = (maxx - minx) > (maxy - miny) ? (maxx - minx) : (maxy - miny);
  length = (maxz - minz) > length ? (maxz - minz) : length;
  pt.n = n;
  if (!build_octree(pt.t, n, ctr.data(), depth, height, minx, miny, minz, length, pt.order))
    return false;
  std::vector<double> vt(9 * (size_t)n);
  for (int i = 0; i < n; i++) memcpy(&vt[9 * (size_t)i], &vtx[9 * (size_t)pt.order[i]], 9 * sizeof(double));
  octree_boxes_panels(pt.t, vt.data());
  octree_neighbours(pt.t, sep_ratio);
  Octree &t = pt.t;

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
