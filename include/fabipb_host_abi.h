/*
 * fabipb_host_abi.h -- memory layout of the reference host's panel, cube and
 * system records, as the plugin ABI passes them (struct ssystem *).
 *
 * The reference defines these in include/gk.h:5-157; a drop-in backend has to
 * read the very same bytes, so the field order and types below are dictated by
 * that interface and must stay identical.  Only the fields the backend reads
 * are documented; the rest are kept for layout.
 */
#ifndef FABIPB_HOST_ABI_H
#define FABIPB_HOST_ABI_H

#ifdef __cplusplus
extern "C" {
#endif

struct panel {
  double vtx[3][3];     /* vertices */
  double a[3][3];       /* edges a[0]=v2-v1, a[1]=v0-v2, a[2]=v1-v0 */
  double x[3];          /* centroid */
  double normal[3];     /* unit normal */
  double nrm[3][3];     /* vertex normals */
  double area;
  double area2;
  int shape;
  int nSurf;            /* 1-based mesh face number */
  int idx;              /* position in the unknown vectors (tree order) */
  struct cube *cube;
  struct panel *next;   /* input order */
  struct panel *nextC;  /* tree order */
};

struct cube {
  int level;
  int i, j, k;
  int flatIdx;          /* FMM index */
  int leafFlatIdx;
  double x[3];          /* expansion centre (enclosing-box centre) */
  int nPnls;
  struct panel *pnls;
  int nNbrs;
  int n2Nbrs;
  struct cube **nbrs;
  int nKids;
  int nthKid;
  struct cube *kids[8];
  struct cube *parent;
  double *mom_pot;
  double *mom_dpdn;
  double *lec_k1;
  double *lec_k2;
  double *lec_k3;
  double *lec_k4;
  double eBoxLo[3];
  double eBoxUp[3];
  double eRad;
  struct cube *next;
  double *mom_chr;
  int *chgIdx;
  int nChgs;
};

struct ssystem {
  int depth;
  int height;
  int maxOrder;
  int nPnls;
  int nChar;
  int nVtxs;
  int nKerl;
  int layer;
  int *ordMom;
  int *ordM2L;
  int *nMom;
  int maxSngs;
  int max1Nbrs;
  int maxQuadOrder;
  double maxSepRatio;
  double *pos, *chr;
  int mesh_flag;
  int benchmarkMode;
  int gpuMode;
  int debugCompareApply;
  int debugComparePrecond;
  int matvecMode;
  int gpuQ2MMode;
  int gpuNearfieldMode;
  int precondCacheMode;
  int nLeafCubesFlat;
  int *leafPanelStart;
  int *leafPanelCount;
  int nNearPairsFlat;
  int *nearPairSrc;
  int *nearPairDst;
  int *nearLeafPairOffset;
  int nFmmCubesFlat;
  struct cube **fmmCubeByIdx;
  int nM2LPairsFlat;
  int *m2lPairSrc;
  int *m2lPairDst;
  int *m2lPairOrder;
  int nM2LDstGroups;
  int *m2lDstGroupStart;
  int *m2lDstGroupCount;
  struct panel **panelByIdx;
  double *panelArea;
  int *fmmLevelStart;
  int *fmmLevelCount;
  int maxlevCudes;
  int maxlevnPnls;
  struct panel *pnlLst;
  struct panel *pnlOLst;
  struct cube **cubeList;
  int chgDepth;
  struct cube **chgCubeList;
};

#ifdef __cplusplus
}
#endif
#endif
