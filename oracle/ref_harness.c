/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (a checker, never shipped).
 *
 * Drives the unmodified reference CPU solver, compiled from its own sources
 * into oracle/_ref/, through its internal entry points, and writes what it
 * computes as raw little-endian binary files so the parity tests can compare
 * the CUDA library with the reference itself:
 *
 *   tree    panel order, leaf layout, near and M2L pair lists, FMM cube data
 *   matvec  one MtVmain (fabipb.c:1237) on a given density
 *   near    the near field alone, applyNearfield1 (fmm.c:679)
 *   rhs     setupRHS (fabipb.c:744)
 *   energy  applyPanelChargeTreeEnergy (treecode.c:927) on a given density
 *   time    wall time of K calls of MtVmain, printed as one JSON line
 *   sample  estimated MtVmain time of a mesh too large to time in full: the
 *           FMM passes timed whole, the near field timed on a leaf sample and
 *           scaled by panel pairs (one JSON line)
 *
 * The setup sequence mirrors main() in fabipb.c:830-1047: defaults, options,
 * loadPanel, the auto policy, gkInit, setupFMM.
 *
 * usage: ref_harness <mode> <mesh-base> <out-prefix> [reference options]
 *        [--sigma=<file of 2N doubles>] [--reps=K] [--warmup=W]
 *
 * Linked with the reference's CUDA backend instead of its stub (ref_harness_gpu,
 * `make refgpu`), option -g=1 runs the same entry points through that backend.
 */

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <sys/time.h>
#include "gkGlobal.h"
#include "gk.h"
#include "fabipb_options.h"

extern ssystem *sys;
extern double kappa, epsilon, epsilon1, epsilon2;
extern int orderMom;

panel *loadPanel(char *panelfile, const char *meshParam, int *numSing, ssystem *sys,
                 const char *meshControlName, double meshControlValue,
                 const char *backendParamName, double backendParamValue);
void gkInit(ssystem *sys, panel *pnlList, int order, int orderMom);
void setupFMM(ssystem *sys);
void applyNearfield1(ssystem *sys, double *alpha, double *sgm, double *beta, double *pot);
int MtVmain(double *alpha, double *sgm, double *beta, double *pot);
void setupRHS(ssystem *sys, double *sgm);
void buildChargeTree(ssystem *sys);
void computeChgMoments(ssystem *sys);
void applyPanelChargeTreeEnergy(ssystem *sys, double *sgm, double *pot);

static double now(void) {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

static void dump(const char *prefix, const char *name, const void *p, size_t bytes) {
  char path[1024];
  FILE *fp;
  snprintf(path, sizeof(path), "%s.%s.bin", prefix, name);
  fp = fopen(path, "wb");
  if (fp == NULL) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
  if (bytes > 0 && fwrite(p, 1, bytes, fp) != bytes) { fprintf(stderr, "short write %s\n", path); exit(2); }
  fclose(fp);
}

static double *readDoubles(const char *path, size_t n) {
  FILE *fp = fopen(path, "rb");
  double *v = (double *)malloc(n * sizeof(double));
  if (fp == NULL || v == NULL || fread(v, sizeof(double), n, fp) != n) {
    fprintf(stderr, "cannot read %zu doubles from %s\n", n, path);
    exit(2);
  }
  fclose(fp);
  return v;
}

static const char *optv(const char *a, const char *name) {
  size_t n = strlen(name);
  if (a[0] != '-' || strncmp(a + 1, name, n) != 0 || a[1 + n] != '=') return NULL;
  return a + 2 + n;
}

int main(int argc, char **argv) {
  const char *mode, *out, *sigmaPath = NULL, *v;
  char base[512];
  int order = -1, reps = 3, warmup = 1, nPnls = 0, i;
  double budget = 0.0;
  int sepExplicit = 0, precondExplicit = 0;
  panel *inputLst;

  if (argc < 4) {
    fprintf(stderr, "usage: %s <tree|matvec|near|rhs|energy|time> <mesh-base> <out-prefix> [opts]\n", argv[0]);
    return 2;
  }
  mode = argv[1];
  snprintf(base, sizeof(base), "%s", argv[2]);
  out = argv[3];

  setenv("FABIPB_REUSE_MESH", "1", 1);
  sys = (ssystem *)calloc(1, sizeof(ssystem));
  sys->height = 2; sys->maxSepRatio = 0.8; sys->maxQuadOrder = 1; sys->nKerl = 4;
  sys->depth = 5; sys->mesh_flag = 1; sys->gpuMode = 0; sys->gpuQ2MMode = 0;
  sys->gpuNearfieldMode = -1; sys->precondCacheMode = 3;
  kappa = 0.1257;

  for (i = 4; i < argc; i++) {
    const char *a = argv[i];
    if ((v = optv(a, "S"))) { sys->maxSepRatio = atof(v); sepExplicit = 1; }
    else if ((v = optv(a, "p"))) order = atoi(v);
    else if ((v = optv(a, "pm"))) orderMom = atoi(v);
    else if ((v = optv(a, "q"))) sys->maxQuadOrder = atoi(v);
    else if ((v = optv(a, "t"))) sys->depth = atoi(v);
    else if ((v = optv(a, "H"))) sys->height = atoi(v);
    else if ((v = optv(a, "k"))) kappa = atof(v);
    else if ((v = optv(a, "eps1"))) epsilon1 = atof(v);
    else if ((v = optv(a, "eps2"))) epsilon2 = atof(v);
    else if ((v = optv(a, "P"))) { sys->precondCacheMode = atoi(v); precondExplicit = 1; }
    else if ((v = optv(a, "g"))) { sys->gpuMode = atoi(v); sys->gpuQ2MMode = sys->gpuMode > 0; }
    else if (strncmp(a, "--sigma=", 8) == 0) sigmaPath = a + 8;
    else if (strncmp(a, "--reps=", 7) == 0) reps = atoi(a + 7);
    else if (strncmp(a, "--warmup=", 9) == 0) warmup = atoi(a + 9);
    else if (strncmp(a, "--budget=", 9) == 0) budget = atof(a + 9);
    else { fprintf(stderr, "unknown option %s\n", a); return 2; }
  }
  epsilon = epsilon2 / epsilon1;

  {
    double t0 = now(), t1;
    inputLst = loadPanel(base, "1", &nPnls, sys, "mesh_resolution", 1.0, "msms_density", 1.0);
    fabipb_resolve_auto_solver_policy(sys, 1, precondExplicit, sepExplicit, nPnls);
    sys->pnlOLst = inputLst;
    gkInit(sys, inputLst, order, orderMom);
    setupFMM(sys);
    t1 = now();
    fprintf(stderr, "ref_harness: setup %.3f s panels=%d leaves=%d near=%d m2l=%d cubes=%d\n",
            t1 - t0, sys->nPnls, sys->nLeafCubesFlat, sys->nNearPairsFlat,
            sys->nM2LPairsFlat, sys->nFmmCubesFlat);
  }

  if (strcmp(mode, "tree") == 0) {
    int n = sys->nPnls, nc = sys->nFmmCubesFlat, c;
    int *order_ = (int *)malloc((size_t)n * sizeof(int));
    int *lev = (int *)malloc((size_t)nc * sizeof(int));
    int *cnt = (int *)malloc((size_t)nc * sizeof(int));
    double *ctr = (double *)malloc((size_t)nc * 4 * sizeof(double));
    int hdr[8];
    panel *p;
    for (i = 0, p = sys->pnlLst; p != NULL; p = p->nextC, i++) order_[i] = p->nSurf - 1;
    for (c = 0; c < nc; c++) {
      cube *cb = sys->fmmCubeByIdx[c];
      lev[c] = cb->level; cnt[c] = cb->nPnls;
      ctr[4 * c] = cb->x[0]; ctr[4 * c + 1] = cb->x[1]; ctr[4 * c + 2] = cb->x[2];
      ctr[4 * c + 3] = cb->eRad;
    }
    hdr[0] = n; hdr[1] = sys->nLeafCubesFlat; hdr[2] = sys->nNearPairsFlat;
    hdr[3] = sys->nM2LPairsFlat; hdr[4] = nc; hdr[5] = sys->maxOrder;
    hdr[6] = sys->depth; hdr[7] = sys->height;
    dump(out, "hdr", hdr, sizeof(hdr));
    dump(out, "order", order_, (size_t)n * sizeof(int));
    dump(out, "leafStart", sys->leafPanelStart, (size_t)sys->nLeafCubesFlat * sizeof(int));
    dump(out, "leafCount", sys->leafPanelCount, (size_t)sys->nLeafCubesFlat * sizeof(int));
    dump(out, "nearSrc", sys->nearPairSrc, (size_t)sys->nNearPairsFlat * sizeof(int));
    dump(out, "nearDst", sys->nearPairDst, (size_t)sys->nNearPairsFlat * sizeof(int));
    dump(out, "m2lSrc", sys->m2lPairSrc, (size_t)sys->nM2LPairsFlat * sizeof(int));
    dump(out, "m2lDst", sys->m2lPairDst, (size_t)sys->nM2LPairsFlat * sizeof(int));
    dump(out, "cubeLevel", lev, (size_t)nc * sizeof(int));
    dump(out, "cubeCount", cnt, (size_t)nc * sizeof(int));
    dump(out, "cubeCtr", ctr, (size_t)nc * 4 * sizeof(double));
    dump(out, "area", sys->panelArea, (size_t)n * sizeof(double));
    return 0;
  }

  if (strcmp(mode, "matvec") == 0 || strcmp(mode, "near") == 0 || strcmp(mode, "energy") == 0) {
    int n2 = 2 * sys->nPnls;
    double *sgm, *pot = (double *)calloc((size_t)n2, sizeof(double));
    double alpha = 1.0, beta = 0.0;
    if (sigmaPath == NULL) { fprintf(stderr, "--sigma required\n"); return 2; }
    sgm = readDoubles(sigmaPath, (size_t)n2);
    if (strcmp(mode, "matvec") == 0) {
      MtVmain(&alpha, sgm, &beta, pot);
      dump(out, "pot", pot, (size_t)n2 * sizeof(double));
    } else if (strcmp(mode, "near") == 0) {
      applyNearfield1(sys, &alpha, sgm, &beta, pot);
      dump(out, "pot", pot, (size_t)n2 * sizeof(double));
    } else {
      double e = 0.0;
      buildChargeTree(sys);
      computeChgMoments(sys);
      applyPanelChargeTreeEnergy(sys, sgm, &e);
      dump(out, "energy", &e, sizeof(double));
      printf("{\"energy_raw\": %.17g, \"energy_kcal\": %.17g}\n", e, e * twoPi * 332.0716);
    }
    return 0;
  }

  if (strcmp(mode, "rhs") == 0) {
    int n2 = 2 * sys->nPnls;
    double *rhs = (double *)calloc((size_t)n2, sizeof(double));
    setupRHS(sys, rhs);
    dump(out, "rhs", rhs, (size_t)n2 * sizeof(double));
    return 0;
  }

  if (strcmp(mode, "time") == 0) {
    int n2 = 2 * sys->nPnls, r;
    double *sgm = (double *)malloc((size_t)n2 * sizeof(double));
    double *pot = (double *)calloc((size_t)n2, sizeof(double));
    double alpha = 1.0, beta = 0.0, t0, t1;
    unsigned long long s = 12345ULL;
    for (i = 0; i < n2; i++) {
      s = s * 6364136223846793005ULL + 1442695040888963407ULL;
      sgm[i] = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    }
    for (r = 0; r < warmup; r++) {
      double w0 = now();
      MtVmain(&alpha, sgm, &beta, pot);
      /* with a time budget, cap the timed repetitions by the warm-up cost */
      if (budget > 0.0) {
        int cap = (int)(budget / (now() - w0));
        if (cap < 1) cap = 1;
        if (reps > cap) reps = cap;
      }
    }
    t0 = now();
    for (r = 0; r < reps; r++) MtVmain(&alpha, sgm, &beta, pot);
    t1 = now();
    printf("{\"panels\": %d, \"reps\": %d, \"seconds\": %.6f, \"matvec_per_s\": %.6g}\n",
           sys->nPnls, reps, t1 - t0, reps / (t1 - t0));
    return 0;
  }

  /*
   * sample: the matvec of a mesh too large to time in full on the host, as
   * `reps` estimated steps.  Each step times one whole MtVmain with the near
   * field switched off (nLeafCubesFlat = 0 only shortens the destination-leaf
   * loop of applyNearfield1CPU, fmm.c:631; the FMM passes and the diagonal
   * run in full) and the near field alone (applyNearfield1, fmm.c:679) over
   * the first L destination leaves, and adds that near-field time scaled by
   * (all near panel pairs) / (panel pairs of the L leaves).  L is chosen from
   * a first probe so that the sample takes about --budget seconds per step.
   */
  if (strcmp(mode, "sample") == 0) {
    int n2 = 2 * sys->nPnls, r, nLeaves = sys->nLeafCubesFlat, L = 0, leaf;
    double *sgm = (double *)malloc((size_t)n2 * sizeof(double));
    double *pot = (double *)calloc((size_t)n2, sizeof(double));
    double alpha = 1.0, beta = 0.0, tFar = 0.0, tNear = 0.0, est = 0.0, probe;
    double *cum = (double *)calloc((size_t)nLeaves + 1, sizeof(double));
    unsigned long long s = 12345ULL;
    for (i = 0; i < n2; i++) {
      s = s * 6364136223846793005ULL + 1442695040888963407ULL;
      sgm[i] = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    }
    for (leaf = 0; leaf < nLeaves; leaf++) {
      double src = 0.0;
      int k;
      for (k = sys->nearLeafPairOffset[leaf]; k < sys->nearLeafPairOffset[leaf + 1]; k++)
        src += sys->leafPanelCount[sys->nearPairSrc[k]];
      cum[leaf + 1] = cum[leaf] + src * sys->leafPanelCount[leaf];
    }
    if (budget <= 0.0) budget = 5.0;
    /* probe: leaves up to 2e7 panel pairs, for the rate */
    for (L = 1; L < nLeaves && cum[L] < 2e7; L++) {}
    {
      double t0;
      sys->nLeafCubesFlat = L;
      t0 = now();
      applyNearfield1(sys, &alpha, sgm, &beta, pot);
      probe = now() - t0;
      sys->nLeafCubesFlat = nLeaves;
    }
    {
      double rate = cum[L] / (probe > 1e-6 ? probe : 1e-6), want = rate * budget;
      for (L = 1; L < nLeaves && cum[L] < want; L++) {}
    }
    for (r = 0; r < warmup + reps; r++) {
      double t0, tf, tn;
      sys->nLeafCubesFlat = 0;
      t0 = now();
      MtVmain(&alpha, sgm, &beta, pot);
      tf = now() - t0;
      sys->nLeafCubesFlat = L;
      t0 = now();
      applyNearfield1(sys, &alpha, sgm, &beta, pot);
      tn = now() - t0;
      sys->nLeafCubesFlat = nLeaves;
      if (r >= warmup) {
        tFar += tf;
        tNear += tn;
        est += tf + tn * (cum[nLeaves] / cum[L]);
      }
    }
    printf("{\"panels\": %d, \"reps\": %d, \"seconds\": %.6f, \"matvec_per_s\": %.6g, "
           "\"far_s\": %.6f, \"near_sample_s\": %.6f, \"sample_leaves\": %d, \"leaves\": %d, "
           "\"sample_pairs\": %.0f, \"near_pairs\": %.0f}\n",
           sys->nPnls, reps, tFar + tNear, reps / est, tFar / reps, tNear / reps, L, nLeaves, cum[L],
           cum[nLeaves]);
    return 0;
  }

  fprintf(stderr, "unknown mode %s\n", mode);
  return 2;
}
