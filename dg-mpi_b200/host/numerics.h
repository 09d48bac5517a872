// numerics.h -- host-side basis / quadrature / face tables for tensor-product
// Lagrange hexahedra (the C++ half of the drop-in; it keeps the reference's
// src/numerics conventions and feeds the device kernels 1D tables).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace dgh {

constexpr int kNS = 5;       // conserved variables (rho, rho u, rho v, rho w, rho E)
constexpr int kMaxOrder = 5; // orders with device kernels

// Quadrature-order rules of the reference:
//   hex:  2(order + gorder) + 1, gorder = 1   (src/numerics/quadrature/tools.cpp:7-17)
//   quad: segment order + 2 = 2 order + 3     (quadrilateral.cpp:36-41, segment.cpp:424-426)
//   points per direction: (qorder + 1) / 2 for odd qorder (quadrature/tools.cpp:20-24)
int hex_quadrature_order(int order);
int quad_quadrature_order(int order);
int points_per_direction(int qorder);

// Gauss-Legendre rule with n points on [-1, 1], ascending nodes.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

// Equidistant nodes on [-1, 1] including the end points
// (BasisTools::equidistant_nodes_1D_range, basis/tools.cpp:9-25).
std::vector<double> equidistant_nodes(int nnodes);

// 1D Lagrange values / derivatives at x for the nodes xn.
void lagrange_1d(double x, const std::vector<double>& xn, double* val, double* grad);

// Faces of the reference hexahedron.  Face f lies on the plane
// xi[face_axis(f)] = face_side(f) ? +1 : -1; its quadrature point q = j*m + i
// (face coordinates (s_i, s_j)) sits on the element's tangential GL grid at
// canonical index face_canonical(f, q) = t1*m + t0, where t0 / t1 are the GL
// indices along the lower / higher of the two tangential element axes.  The
// map follows the corner ordering of get_points_on_face_hexahedron
// (src/numerics/basis/shape.cpp:224-324) for orientation 0.
int face_axis(int f);
int face_side(int f);
void face_canonical_map(int m, int f, std::vector<int>& canon);

// Point order of a face seen with orientation `orient`
// (get_face_pts_order_wrt_orient0_hexahedron, shape.cpp:326-428).
void face_orientation_order(int orient, int npts, std::vector<int>& order);

// Unit-cube face corner node lists of the linear geometric basis, in the
// order get_local_nodes_on_face_hexahedron (shape.cpp:430-480) returns them
// for gorder = 1.
std::array<int, 4> face_geometry_nodes(int f);

// 1D tables of order p consumed by the kernels.
struct Tables1D {
    int p = 0, n = 1, m = 2;               // n = p+1 coefficients, m = p+2 GL points
    std::vector<double> xq, wq;            // volume/face GL nodes and weights [m]
    std::vector<double> B, D;              // B[q*n+b] = phi_b(x_q), D = phi_b'(x_q)
    std::vector<double> Minv;              // [n*n] inverse 1D mass matrix
    int me = 0;                            // IC / error rule: 2*max(p,1)+2 points
    std::vector<double> xe, we, Be;        // [me], [me], [me*n]
    int mm = 0;                            // inverse-mass rule: 2p+2 points
    std::vector<double> xm, wm, Bm;        // [mm], [mm], [mm*n]
};
Tables1D make_tables(int p);

// Inverse mass matrix of one trilinear element with nodes X [8][3]
// (helpers.cpp:54-100: the mass matrix B^T diag(w djac) B on the order-2p rule,
// inverted by an unpivoted LU factorisation as BasisTools::get_inv_mass_matrices
// does, basis/tools.cpp:86-110), written transposed: out[k * nb + j] = iMM[j][k].
// Returns false for a singular factorisation.
bool general_inverse_mass(const Tables1D& t, const double* X, double* out);

// Jacobian of the trilinear map of nodes X [8][3] at reference point xi:
// jac[i*3 + j] = sum_n X[n][i] dphi_n/dxi_j (basis/tools.cpp:42-66).
void trilinear_jacobian(const double* X, const double* xi, double* jac);
double det3(const double* M);

}  // namespace dgh
