// temporary: filled in by charges.cu / solver.cu
#include "context.cuh"
namespace fb {
struct ChargeTreeDev {};
struct PrecondDev {};
bool setup_charges(Context &c, int m, const double *pos, const double *q) { set_error("charges: not built yet"); return false; }
void free_charges(Context &c) {}
void free_precond(Context &c) {}
bool launch_rhs(Context &c, int useTree, double *rhs) { set_error("rhs: not built yet"); return false; }
bool launch_energy(Context &c, const double *sgm, double *raw) { set_error("energy: not built yet"); return false; }
bool precond_setup(Context &c, int mode) { set_error("precond: not built yet"); return false; }
bool precond_apply(Context &c, const double *b, double *x) { set_error("precond: not built yet"); return false; }
bool gmres_solve(Context &c, const double *b, double *x, int restart, int maxit, double tol, int *iters, double *resid, int *info) { set_error("solve: not built yet"); return false; }
}
