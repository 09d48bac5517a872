// case.h -- host-side case helpers: L2 projection of an initial condition
// (sum-factorised, OpenMP) and the CFL time step.
#pragma once
#include <vector>

#include "mesh.h"
#include "numerics.h"

namespace dgh {

// Solver::init_state_from_fcn + SolverTools::L2_projection
// (src/solver/base.cpp:113-223, src/solver/tools.cpp:66-122) for affine
// elements: rhs = B_e^T (w * djac * f) on the 2*max(p,1)+2 point rule, then
// U = (M_1^-1 x M_1^-1 x M_1^-1) rhs / djac.  Output Uc[ne][nb][5].
void project_initial_condition(const PreparedMesh& pm, const Tables1D& t, int ic_type, const double* data,
                               double gamma, double R, double time, double* Uc);

// dt = cfl * hmin / ((2p+1) * max_nodes(|u| + c)); the nodal values of an
// equidistant Lagrange basis are its coefficients.  Returns <= 0 on a
// non-physical state.
double cfl_time_step(const PreparedMesh& pm, int p, double gamma, const double* Uc, double cfl);

}  // namespace dgh
