// tree.hpp -- the panel and charge octrees and their flattened layouts.
//
// The octree, its leaf order, its enclosing-box centres and its near and
// interaction lists are a pure function of the panel vertices and (-t, -H, -S),
// and the matvec's summation pattern depends on all of them, so they are
// reproduced exactly:
//   goDown        src/gkSetup.c:142-183  child = ix+2iy+4iz from strict '>'
//                 tests against minx+(i+0.5)*sideLen[level]
//   linkcubes     src/gkSetup.c:194-236  depth-first, children in index order
//   getEnclBoxs   src/gkSetup.c:264-322  centre of the vertex bounding box
//   near          src/gkSetup.c:332-349  far iff (r1+r2)/dist < S
//   getNbrs       src/gkSetup.c:363-437  lists from the parent's near list
//   layouts       src/fmm.c:234-404
// Depth-first order with children in index order is the order of the Morton
// key whose 3-bit digit per level is (iz,iy,ix); points are stable-sorted by
// that key, so inside a leaf they keep input order as goDown appends them.
#pragma once
#include <cstdint>
#include <vector>

namespace fb {

struct Octree {
  int depth = 0, height = 0, nCubes = 0;
  std::vector<int> levStart;                      // depth+2 entries
  std::vector<int> level, parent, kidStart, kidCount, itemStart, itemCount;
  std::vector<double> x, rad, lo, up;             // 3, 1, 3, 3 per cube
  std::vector<int> nbrStart, nNbr1, nNbr2, nbr;   // levels >= height
};

// Build the octree over `pts` (3 doubles each).  `sorted` receives the item
// permutation (tree position -> item index).
bool build_octree(Octree &t, int n, const double *pts, int depth, int height, double minx,
                  double miny, double minz, double length, std::vector<int> &sorted);
// enclosing boxes from panel vertices (vtx in tree order, 9 per panel)
void octree_boxes_panels(Octree &t, const double *vtx_tree);
// enclosing boxes from points (pts in original order, `sorted` permutation)
void octree_boxes_points(Octree &t, const double *pts, const std::vector<int> &sorted);
void octree_neighbours(Octree &t, double eta0);

struct PanelTree {
  Octree t;
  int n = 0;
  std::vector<int> order;      // tree index -> input index
  // flattened layouts of the reference
  int nLeaves = 0;
  std::vector<int> leafStart, leafCount, leafCube;
  std::vector<int> nearOff, nearSrc, nearDst;  // CSR by destination leaf
  int nFmm = 0;
  std::vector<int> fmmCube, cubeFmm;           // flat FMM index <-> cube id
  std::vector<int> fmmLevelStart, fmmLevelCount;
  std::vector<int> m2lOff, m2lSrc;             // CSR by destination FMM cube
  std::vector<int> m2lPairSrc, m2lPairDst;     // reference pair order
  // expansion orders (src/gkSetup.c:42-81)
  int maxOrder = 0;
  std::vector<int> ordMom, ordM2L;
};

bool build_panel_tree(PanelTree &pt, int n, const double *vtx, int depth, int height,
                      double sep_ratio, int order, int order_mom);
// the expansion orders and the flattened layouts (near pairs by leaf, FMM
// cube order, M2L lists) from a finished octree and panel order
bool finish_panel_tree(PanelTree &pt, int order, int order_mom);

}  // namespace fb
