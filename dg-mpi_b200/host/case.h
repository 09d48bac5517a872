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
// U = (M_1^-1 x M_1^-1 x M_1^-1) rhs / djac.  Output Uc[e_end-e_begin][nb][5]
// for the elements [e_begin, e_end) (e_end < 0: all).
void project_initial_condition(const PreparedMesh& pm, const Tables1D& t, int ic_type, const double* data,
                               double gamma, double R, double time, double* Uc, int e_begin = 0, int e_end = -1);

// dt = cfl * hmin / ((2p+1) * max_nodes(|u| + c)); the nodal values of an
// equidistant Lagrange basis are its coefficients.  Returns <= 0 on a
// non-physical state.  Uc holds the elements [e_begin, e_end) (e_end < 0: all)
// and hmin is taken over those elements.
double cfl_time_step(const PreparedMesh& pm, int p, double gamma, const double* Uc, double cfl, int e_begin = 0,
                     int e_end = -1);

// volume and smallest edge length of the elements [e_begin, e_end)
double range_volume(const PreparedMesh& pm, int e_begin, int e_end);
double range_hmin(const PreparedMesh& pm, int e_begin, int e_end);

}  // namespace dgh
