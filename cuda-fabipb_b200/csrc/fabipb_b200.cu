// fabipb_b200.cu -- the library is compiled as one translation unit so the
// constant-memory tables (quadrature rules, multi-index tables) are shared by
// every kernel without relocatable device code.
#include "near.cu"
#include "fmm.cu"
#include "charges.cu"
#include "solver.cu"
#include "tree_dev.cu"
#include "api.cu"
#include "abi.cu"
#include "adjoint.cu"
#include "noalloc.cu"
#include "peak.cu"
