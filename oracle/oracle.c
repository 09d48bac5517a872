/*
 * oracle.c -- CPU restatement of DG-MPI's 3D Euler residual + RK4 hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Plain C99 + OpenMP, written from
 * the reference's algorithm; every block cites the reference file:line it
 * follows (paths relative to the reference project root).  It deliberately
 * keeps the reference's dense per-element formulation (dense B*U, per-qp
 * geometry, dense inverse mass) so that it stands for the reference's Kokkos
 * OpenMP build both as parity oracle and as timed CPU baseline.
 *
 * Third-party arithmetic: kokkos-kernels (submodule externals/kokkos-kernels,
 * pinned commit not recoverable -- the submodule is empty) supplies
 * KokkosBatched::{Serial,Team}Gemm<Algo::Gemm::Unblocked> (plain triple-loop
 * GEMM), {Serial,Team}LU<Algo::LU::Unblocked> (Doolittle LU without
 * pivoting) + SolveLU, and KokkosBlas::{axpy,update,fill}.  Those published
 * semantics are restated below as plain loops.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NS ORC_NS

/* ------------------------------------------------------------------------ */
/* quadrature                                                                */
/* ------------------------------------------------------------------------ */

/* QuadratureTools::get_gausslegendre_quadrature_order, quadrature/tools.cpp:7-17
 * (hex; gorder hard-coded to 1) */
int orc_hex_quadrature_order(int order) { return 2 * (order + 1) + 1; }

/* SegmentQuadrature::get_gausslegendre_quadrature_order, segment.cpp:424-426 */
int orc_segment_quadrature_order(int order) { return 2 * order + 1; }

/* QuadrilateralQuadrature::get_gausslegendre_quadrature_order,
 * quadrilateral.cpp:36-41: segment order + 2 */
int orc_quad_quadrature_order(int order) { return orc_segment_quadrature_order(order) + 2; }

/* QuadratureTools::get_number_of_quadrature_points, quadrature/tools.cpp:20-24 */
int orc_num_quadrature_points_1d(int qorder)
{
    int nq1 = 0;
    if ((qorder + 2) % 2 == 0) nq1 = (qorder + 2) / 2;
    if ((qorder + 1) % 2 == 0) nq1 = (qorder + 1) / 2;
    return nq1;
}

/* Gauss-Legendre nodes (ascending) and weights for the rule of quadrature
 * order `qorder`.  The reference tabulates them to 32 digits
 * (numerics/nodes.cpp:97-~500, quadrature/segment.cpp:7-~420); here they are
 * computed by Newton iteration on P_n in long double and rounded once, which
 * reproduces the correctly-rounded table values (pinned by a golden test). */
void orc_gauss_legendre_1d(int qorder, double* pts, double* wts)
{
    int n = orc_num_quadrature_points_1d(qorder);
    for (int i = 0; i < (n + 1) / 2; i++) {
        long double z = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
        long double dp = 1.0L;
        for (int it = 0; it < 200; it++) {
            long double p0 = 1.0L, p1 = z;
            for (int k = 2; k <= n; k++) {
                long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1.0L; }
            dp = n * (z * p1 - p0) / (z * z - 1.0L);
            long double dz = p1 / dp;
            z -= dz;
            if (fabsl(dz) < 1e-30L) break;
        }
        {   /* final derivative at the converged root */
            long double p0 = 1.0L, p1 = z;
            for (int k = 2; k <= n; k++) {
                long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0L);
        }
        long double w = 2.0L / ((1.0L - z * z) * dp * dp);
        if (2 * i + 1 == n) z = 0.0L;
        pts[n - 1 - i] = (double)z;
        pts[i] = -(double)z;
        wts[i] = (double)w;
        wts[n - 1 - i] = (double)w;
    }
}

/* HexahedronQuadrature::get_quadrature_gauss_legendre, hexahedron.cpp:6-36:
 * point index k*n*n + j*n + i, x fastest; weight w_i*w_j*w_k */
static int hex_quadrature(int qorder, double** pts, double** wts)
{
    int n = orc_num_quadrature_points_1d(qorder);
    double* x = malloc(sizeof(double) * n);
    double* w = malloc(sizeof(double) * n);
    orc_gauss_legendre_1d(qorder, x, w);
    int nq = n * n * n;
    *pts = malloc(sizeof(double) * nq * 3);
    *wts = malloc(sizeof(double) * nq);
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                int q = k * n * n + j * n + i;
                (*pts)[q * 3 + 0] = x[i];
                (*pts)[q * 3 + 1] = x[j];
                (*pts)[q * 3 + 2] = x[k];
                (*wts)[q] = w[i] * w[j] * w[k];
            }
    free(x);
    free(w);
    return nq;
}

/* QuadrilateralQuadrature::get_quadrature_gauss_legendre, quadrilateral.cpp:7-34 */
static int quad_quadrature(int qorder, double** pts, double** wts)
{
    int n = orc_num_quadrature_points_1d(qorder);
    double* x = malloc(sizeof(double) * n);
    double* w = malloc(sizeof(double) * n);
    orc_gauss_legendre_1d(qorder, x, w);
    int nq = n * n;
    *pts = malloc(sizeof(double) * nq * 2);
    *wts = malloc(sizeof(double) * nq);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            (*pts)[(j * n + i) * 2 + 0] = x[i];
            (*pts)[(j * n + i) * 2 + 1] = x[j];
            (*wts)[j * n + i] = w[i] * w[j];
        }
    free(x);
    free(w);
    return nq;
}

/* ------------------------------------------------------------------------ */
/* Lagrange basis on equidistant nodes                                       */
/* ------------------------------------------------------------------------ */

/* BasisTools::equidistant_nodes_1D_range, basis/tools.cpp:9-25 */
void orc_equidistant_nodes(double start, double stop, int n, double* x)
{
    if (n <= 1) { x[0] = 0.0; return; }
    double dx = (stop - start) / ((double)n - 1.0);
    for (int i = 0; i < n; i++) x[i] = start + (double)i * dx;
}

/* get_lagrange_basis_val_1D, basis/tools.cpp:114-127 */
void orc_lagrange_1d_val(double x, int nn, const double* xn, double* phi)
{
    for (int i = 0; i < nn; i++) {
        phi[i] = 1.0;
        for (int j = 0; j < nn; j++) {
            if (i == j) continue;
            phi[i] *= (x - xn[j]) / (xn[i] - xn[j]);
        }
    }
}

/* get_lagrange_basis_grad_1D, basis/tools.cpp:129-149 */
void orc_lagrange_1d_grad(double x, int nn, const double* xn, double* gphi)
{
    for (int i = 0; i < nn; i++) {
        gphi[i] = 0.0;
        for (int j = 0; j < nn; j++) {
            if (i == j) continue;
            double prod = 1.0;
            for (int k = 0; k < nn; k++) {
                if (i == k) continue;
                else if (j == k) prod *= 1.0 / (xn[i] - xn[k]);
                else prod *= (x - xn[k]) / (xn[i] - xn[k]);
            }
            gphi[i] += prod;
        }
    }
}

/* Basis::get_values for LagrangeHex, basis.cpp:93-111 + basis/tools.cpp:215-247:
 * basis index k(p+1)^2 + j(p+1) + i, value valx*valy*valz.  val[nq][nb] */
void orc_lagrange_hex_val(int p, int nq, const double* xq, double* val)
{
    int n = p + 1, nb = n * n * n;
    if (p == 0) { for (int q = 0; q < nq; q++) val[q] = 1.0; return; }
    double xn[16], vx[16], vy[16], vz[16];
    orc_equidistant_nodes(-1.0, 1.0, n, xn);
    for (int q = 0; q < nq; q++) {
        orc_lagrange_1d_val(xq[q * 3 + 0], n, xn, vx);
        orc_lagrange_1d_val(xq[q * 3 + 1], n, xn, vy);
        orc_lagrange_1d_val(xq[q * 3 + 2], n, xn, vz);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++)
                    val[q * nb + k * n * n + j * n + i] = vx[i] * vy[j] * vz[k];
    }
}

/* Basis::get_grads for LagrangeHex, basis.cpp:113-128 + basis/tools.cpp:249-295.
 * grad[nq][nb][3]; for p == 0 the reference leaves the (zeroed) view unset. */
void orc_lagrange_hex_grad(int p, int nq, const double* xq, double* grad)
{
    int n = p + 1, nb = n * n * n;
    if (p == 0) { for (int q = 0; q < nq * 3; q++) grad[q] = 0.0; return; }
    double xn[16], vx[16], vy[16], vz[16], gx[16], gy[16], gz[16];
    orc_equidistant_nodes(-1.0, 1.0, n, xn);
    for (int q = 0; q < nq; q++) {
        orc_lagrange_1d_val(xq[q * 3 + 0], n, xn, vx);
        orc_lagrange_1d_val(xq[q * 3 + 1], n, xn, vy);
        orc_lagrange_1d_val(xq[q * 3 + 2], n, xn, vz);
        orc_lagrange_1d_grad(xq[q * 3 + 0], n, xn, gx);
        orc_lagrange_1d_grad(xq[q * 3 + 1], n, xn, gy);
        orc_lagrange_1d_grad(xq[q * 3 + 2], n, xn, gz);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    double* g = grad + ((size_t)q * nb + k * n * n + j * n + i) * 3;
                    g[0] = gx[i] * vy[j] * vz[k];
                    g[1] = vx[i] * gy[j] * vz[k];
                    g[2] = vx[i] * vy[j] * gz[k];
                }
    }
}

/* LagrangeQuad gradients (order 1 face geometry basis), basis/tools.cpp:179-213.
 * grad[nq][nb][2] */
static void lagrange_quad_grad(int p, int nq, const double* xq /*[nq][2]*/, double* grad)
{
    int n = p + 1, nb = n * n;
    double xn[16], vx[16], vy[16], gx[16], gy[16];
    orc_equidistant_nodes(-1.0, 1.0, n, xn);
    for (int q = 0; q < nq; q++) {
        orc_lagrange_1d_val(xq[q * 2 + 0], n, xn, vx);
        orc_lagrange_1d_val(xq[q * 2 + 1], n, xn, vy);
        orc_lagrange_1d_grad(xq[q * 2 + 0], n, xn, gx);
        orc_lagrange_1d_grad(xq[q * 2 + 1], n, xn, gy);
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                grad[(q * nb + j * n + i) * 2 + 0] = gx[i] * vy[j];
                grad[(q * nb + j * n + i) * 2 + 1] = vx[i] * gy[j];
            }
    }
}

/* ------------------------------------------------------------------------ */
/* hexahedron faces                                                          */
/* ------------------------------------------------------------------------ */

/* get_points_on_face_hexahedron, basis/shape.cpp:224-324 */
void orc_points_on_face(int face, int orient, int np, const double* fpts, double* epts)
{
    static const double xr[8] = {-1., 1., -1., 1., -1., 1., -1., 1.};
    static const double yr[8] = {-1., -1., 1., 1., -1., -1., 1., 1.};
    static const double zr[8] = {-1., -1., -1., -1., 1., 1., 1., 1.};
    static const int corners[6][4] = {
        {0, 2, 3, 1}, {0, 1, 5, 4}, {1, 3, 7, 5}, {3, 2, 6, 7}, {2, 0, 4, 6}, {4, 5, 7, 6}};
    int node[4];
    int cycle = orient % 4, flip = orient / 4;
    for (int j = 0; j < 4; j++) node[j] = corners[face][(j + cycle) % 4];
    if (flip >= 1) { int t = node[1]; node[1] = node[3]; node[3] = t; }
    double xe[4], ye[4], ze[4], b[4];
    for (int j = 0; j < 4; j++) { xe[j] = xr[node[j]]; ye[j] = yr[node[j]]; ze[j] = zr[node[j]]; }
    for (int i = 0; i < np; i++) {
        double xb = (fpts[i * 2 + 0] + 1.) / 2.;
        double yb = (fpts[i * 2 + 1] + 1.) / 2.;
        b[0] = (1. - xb) * (1. - yb);
        b[1] = xb * (1. - yb);
        b[2] = xb * yb;
        b[3] = (1. - xb) * yb;
        epts[i * 3 + 0] = 0.0; epts[i * 3 + 1] = 0.0; epts[i * 3 + 2] = 0.0;
        for (int j = 0; j < 4; j++) {
            epts[i * 3 + 0] += b[j] * xe[j];
            epts[i * 3 + 1] += b[j] * ye[j];
            epts[i * 3 + 2] += b[j] * ze[j];
        }
    }
}

/* get_face_pts_order_wrt_orient0_hexahedron, basis/shape.cpp:326-428 */
void orc_face_pts_order(int orient, int npts, int* order)
{
    int n1 = (int)(sqrt((double)npts) + 0.5);
    int np1 = npts + 1;
    switch (orient) {
    case 0:
        for (int i = 0; i < npts; i++) order[i] = i;
        break;
    case 1: {
        int curr = n1 - 1;
        for (int i = 0; i < npts; i++) { order[i] = curr; curr = (curr + n1) % np1; }
        break;
    }
    case 2:
        for (int i = 0; i < npts; i++) order[i] = npts - 1 - i;
        break;
    case 3: {
        int curr = npts - n1;
        for (int i = 0; i < npts; i++) { order[i] = curr; curr -= n1; if (curr < 0) curr += np1; }
        break;
    }
    case 4: {
        int curr = 0;
        for (int i = 0; i < npts; i++) { order[i] = curr; curr += n1; if (curr >= npts) curr -= npts - 1; }
        break;
    }
    case 5: {
        int curr = n1 - 1, k = 0;
        for (int i = 0; i < n1; i++) {
            for (int j = 0; j < n1; j++) { order[k] = curr; curr -= 1; k += 1; }
            curr += 2 * n1;
        }
        break;
    }
    case 6: {
        int curr = npts - 1;
        for (int i = 0; i < npts; i++) { order[i] = curr; curr -= n1; if (curr < 0) curr += npts - 1; }
        break;
    }
    case 7: {
        int curr = npts - n1, k = 0;
        for (int i = 0; i < n1; i++) {
            for (int j = 0; j < n1; j++) { order[k] = curr; curr += 1; k += 1; }
            curr -= 2 * n1;
        }
        break;
    }
    default:
        for (int i = 0; i < npts; i++) order[i] = -1;
    }
}

/* get_local_nodes_on_face_hexahedron, basis/shape.cpp:430-480 */
void orc_local_nodes_on_face(int face, int gorder, int* lf)
{
    int i0 = 0, d0 = 0, d1 = 0, g1 = gorder + 1;
    switch (face) {
    case 0: i0 = 0; d0 = g1; d1 = 1; break;
    case 1: i0 = 0; d0 = 1; d1 = g1 * g1; break;
    case 2: i0 = gorder; d0 = g1; d1 = g1 * g1; break;
    case 3: i0 = g1 * g1 - 1; d0 = -1; d1 = g1 * g1; break;
    case 4: i0 = gorder * g1; d0 = -g1; d1 = g1 * g1; break;
    case 5: i0 = gorder * g1 * g1; d0 = 1; d1 = g1; break;
    }
    for (int j = 0, k = 0; j < g1; j++)
        for (int i = 0; i < g1; i++, k++) lf[k] = i0 + i * d0 + j * d1;
}

/* ------------------------------------------------------------------------ */
/* physics (pointwise)                                                       */
/* ------------------------------------------------------------------------ */

/* EulerFcnType::get_pressure<3>, euler/functions.cpp:10-23 */
double orc_pressure(double gamma, const double* U)
{
    double rKE = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
    return (gamma - 1.0) * (U[4] - 0.5 * rKE);
}

/* EulerFcnType::get_maxwavespeed<3>, euler/functions.cpp:25-40 */
double orc_maxwavespeed(double gamma, const double* U)
{
    double rho1 = 1. / U[0];
    double sqrtrKE = sqrt(U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * rho1;
    return sqrtrKE + sqrt(gamma * orc_pressure(gamma, U) * rho1);
}

/* EulerFcnType::conv_flux_interior<3>, euler/functions.cpp:64-91;
 * Fdir[j*5 + s] = flux of state s in direction j */
void orc_conv_flux(double gamma, const double* U, double* F)
{
    const double r1 = 1. / U[0];
    const double ru = U[1], rv = U[2], rw = U[3], rE = U[4];
    const double P = orc_pressure(gamma, U);
    F[0] = ru;
    F[1] = ru * ru * r1 + P;
    F[2] = ru * rv * r1;
    F[3] = ru * rw * r1;
    F[4] = (rE + P) * ru * r1;
    F[5] = rv;
    F[6] = rv * ru * r1;
    F[7] = rv * rv * r1 + P;
    F[8] = rv * rw * r1;
    F[9] = (rE + P) * rv * r1;
    F[10] = rw;
    F[11] = rw * ru * r1;
    F[12] = rw * rv * r1;
    F[13] = rw * rw * r1 + P;
    F[14] = (rE + P) * rw * r1;
}

/* BaseConvNumFluxType::compute_flux_laxfriedrichs<3>, base/functions.cpp:33-89 */
static void flux_lf(double gamma, const double* UL, const double* UR, const double* N, double* F)
{
    double n_hat[3], n_mag = 0.0;
    for (int d = 0; d < 3; d++) n_mag += N[d] * N[d];
    n_mag = sqrt(n_mag);
    for (int d = 0; d < 3; d++) n_hat[d] = N[d] / n_mag;
    double Fq[15], dU[NS], FqL[NS] = {0}, FqR[NS] = {0};
    orc_conv_flux(gamma, UL, Fq);
    for (int s = 0; s < NS; s++)
        for (int d = 0; d < 3; d++) FqL[s] += Fq[s + d * NS] * n_hat[d];
    orc_conv_flux(gamma, UR, Fq);
    for (int s = 0; s < NS; s++)
        for (int d = 0; d < 3; d++) FqR[s] += Fq[s + d * NS] * n_hat[d];
    for (int s = 0; s < NS; s++) dU[s] = UR[s] - UL[s];
    double a = orc_maxwavespeed(gamma, UL);
    double aR = orc_maxwavespeed(gamma, UR);
    if (aR > a) a = aR;
    for (int s = 0; s < NS; s++) F[s] = n_mag * (0.5 * (FqL[s] + FqR[s]) - 0.5 * a * dU[s]);
}

/* EulerConvNumFluxType::compute_flux_hllc<3>, euler/functions.cpp:298-399.
 * The reference prints and asserts on the fall-through branch; here it
 * reports -1 and returns zero flux. */
static int flux_hllc(double gam, const double* UL, const double* UR, const double* N, double* F)
{
    const double djac = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    const double djac1 = 1. / djac;
    const double n[3] = {N[0] * djac1, N[1] * djac1, N[2] * djac1};
    const double rhoL = UL[0], rhoL1 = 1. / rhoL;
    const double unL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) * rhoL1;
    const double PL = orc_pressure(gam, UL);
    const double aL = sqrt(gam * PL * rhoL1);
    const double rhoR = UR[0], rhoR1 = 1. / rhoR;
    const double unR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) * rhoR1;
    const double PR = orc_pressure(gam, UR);
    const double aR = sqrt(gam * PR * rhoR1);
    const double rAvg = 0.5 * (rhoL + rhoR);
    const double aAvg = 0.5 * (aL + aR);
    const double pStar = fmax(0., 0.5 * (PL + PR - (unR - unL) * rAvg * aAvg));
    double qL = 1.0, qR = 1.0;
    if (pStar / PL > 1.) qL = sqrt(1. + (gam + 1.) / (2. * gam) * (pStar / PL - 1.));
    if (pStar / PR > 1.) qR = sqrt(1. + (gam + 1.) / (2. * gam) * (pStar / PR - 1.));
    const double sL = unL - aL * qL;
    const double sR = unR + aR * qR;
    const double sStar = (PR - PL + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR)) /
                         (rhoL * (sL - unL) - rhoR * (sR - unR));
    if (sL >= 0.) {
        F[0] = djac * rhoL * unL;
        for (int i = 0; i < 3; i++) F[1 + i] = djac * (UL[1 + i] * unL + PL * n[i]);
        F[4] = djac * ((UL[4] + PL) * unL);
    } else if (sR <= 0.) {
        F[0] = djac * rhoR * unR;
        for (int i = 0; i < 3; i++) F[1 + i] = djac * (UR[1 + i] * unR + PR * n[i]);
        F[4] = djac * (UR[4] + PR) * unR;
    } else if ((sL < 0.) && (sStar >= 0.)) {
        const double c = (sL - unL) / (sL - sStar);
        const double f1 = sStar - unL;
        const double f2 = sStar + PL / (rhoL * (sL - unL));
        F[0] = djac * (rhoL * unL + rhoL * sL * (c - 1.));
        for (int i = 0; i < 3; i++)
            F[1 + i] = djac * (UL[1 + i] * unL + PL * n[i] + sL * (UL[1 + i] * (c - 1.) + rhoL * c * f1 * n[i]));
        F[4] = djac * ((UL[4] + PL) * unL + sL * (UL[4] * (c - 1.) + rhoL * c * f1 * f2));
    } else if ((sStar < 0.) && (sR > 0.)) {
        const double c = (sR - unR) / (sR - sStar);
        const double f1 = sStar - unR;
        const double f2 = sStar + PR / (rhoR * (sR - unR));
        F[0] = djac * (rhoR * unR + rhoR * sR * (c - 1.));
        for (int i = 0; i < 3; i++)
            F[1 + i] = djac * (UR[1 + i] * unR + PR * n[i] + sR * (UR[1 + i] * (c - 1.) + rhoR * c * f1 * n[i]));
        F[4] = djac * ((UR[4] + PR) * unR + sR * (UR[4] * (c - 1.) + rhoR * c * f1 * f2));
    } else {
        for (int s = 0; s < NS; s++) F[s] = 0.0;
        return -1;
    }
    return 0;
}

/* Physics<3>::get_conv_flux_numerical dispatch, physics/base/base.cpp:48-62 */
int orc_num_flux(int flux_type, double gamma, const double* UL, const double* UR,
                 const double* N, double* F)
{
    if (flux_type == ORC_FLUX_HLLC) return flux_hllc(gamma, UL, UR, N, F);
    flux_lf(gamma, UL, UR, N, F);
    return 0;
}

/* Initial conditions / exact solutions (physics/base/base.cpp:90-137) */
void orc_ic_eval(int ic, int ndata, const double* data, double gamma, double R,
                 const double* x, double t, double* U)
{
    const double PI = 3.14159265358979323846;
    (void)ndata;
    if (ic == ORC_IC_UNIFORM) {
        /* set_state_uniform_3D, physics/base/base.cpp:150-158 */
        for (int s = 0; s < NS; s++) U[s] = data[s];
    } else if (ic == ORC_IC_SPHERE) {
        /* set_smooth_sphere, physics/base/base.cpp:177-194 */
        double magR = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        for (int s = 0; s < NS; s++) U[s] = 0.5 * (1. - 0.) * (tanh(PI * (0.5 - magR) / 0.5) + 1.0) + 0.;
    } else if (ic == ORC_IC_VORTEX_REF) {
        /* set_state_isentropic_vortex (3D), euler/functions.cpp:147-191 */
        double rho0 = 1., sos0 = 1., L = 1., Mach = 1.0, radius = L / 10., sigma = 1;
        double beta = Mach * 5. * sqrt(2.) / (4. * PI) * exp(0.5);
        double u0 = Mach * sos0;
        double x1 = x[0] - 0.5, y1 = x[2] - 0.5;
        double f = -0.5 / (sigma * sigma) * (x1 * x1 + y1 * y1) / (radius * radius);
        double Omega = beta * exp(f);
        double du = -y1 / radius * Omega, dv = x1 / radius * Omega;
        double dT = -(gamma - 1.) / 2. * Omega * Omega;
        double p = 1. / gamma * pow(1 + dT, gamma / (gamma - 1.));
        U[0] = pow(rho0 + dT, 1. / (gamma - 1.));
        U[1] = U[0] * (u0 + du);
        U[2] = 0.;
        U[3] = U[0] * dv;
        double rKE = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
        U[4] = p / (gamma - 1.0) + 0.5 * rKE;
    } else if (ic == ORC_IC_VORTEX_XY) {
        /* 2D isentropic vortex, euler/functions.cpp:94-145, extruded in z,
         * centred at (xc, yc) and advected with (ub, vb) on a periodic box */
        double rhob = data[0], ub = data[1], vb = data[2], pb = data[3], vs = data[4];
        double xc = data[5], yc = data[6], Lx = data[7], Ly = data[8];
        double Tb = pb / (rhob * R);
        double s = pb / pow(rhob, gamma);
        double xr = x[0] - xc - ub * t;
        double yr = x[1] - yc - vb * t;
        xr -= Lx * floor(xr / Lx + 0.5);
        yr -= Ly * floor(yr / Ly + 0.5);
        double r = sqrt(xr * xr + yr * yr);
        double r2 = r * r;
        double dUm = vs / (2.0 * PI) * exp(0.5 * (1.0 - r2));
        double du = dUm * -1.0 * yr, dv = dUm * xr;
        double dT = -1.0 * (gamma - 1.0) * (vs * vs) / (8.0 * gamma * (PI * PI)) * exp(1.0 - r2);
        double u = ub + du, v = vb + dv, T = Tb + dT;
        double rho = pow(T / s, 1.0 / (gamma - 1.0));
        double rhou = rho * u, rhov = rho * v;
        U[0] = rho;
        U[1] = rhou;
        U[2] = rhov;
        U[3] = 0.0;
        U[4] = rho * R / (gamma - 1.0) * T + 0.5 * (rhou * rhou + rhov * rhov) / rho;
    } else if (ic == ORC_IC_TAYLOR_GREEN) {
        double M = data[0];
        double u = sin(x[0]) * cos(x[1]) * cos(x[2]);
        double v = -cos(x[0]) * sin(x[1]) * cos(x[2]);
        double p = 1.0 / (gamma * M * M) + (cos(2.0 * x[0]) + cos(2.0 * x[1])) * (cos(2.0 * x[2]) + 2.0) / 16.0;
        U[0] = 1.0;
        U[1] = u;
        U[2] = v;
        U[3] = 0.0;
        U[4] = p / (gamma - 1.0) + 0.5 * (u * u + v * v);
    } else {
        for (int s = 0; s < NS; s++) U[s] = 0.0;
    }
}

/* ------------------------------------------------------------------------ */
/* small dense linear algebra (Math::*, math/linear_algebra.cpp)             */
/* ------------------------------------------------------------------------ */

/* Math::det for 3x3, linear_algebra.cpp:243-259 */
static double det3(const double* m)
{
#define M(i, j) m[(i) * 3 + (j)]
    return M(0, 0) * M(1, 1) * M(2, 2) - M(0, 0) * M(1, 2) * M(2, 1) - M(0, 1) * M(1, 0) * M(2, 2) +
           M(0, 1) * M(1, 2) * M(2, 0) + M(0, 2) * M(1, 0) * M(2, 1) - M(0, 2) * M(1, 1) * M(2, 0);
}

/* Math::invA closed form for dim == 3, linear_algebra.cpp:108-122 */
static void inv3(const double* m, double* im)
{
    double det = det3(m);
#define IM(i, j) im[(i) * 3 + (j)]
    IM(0, 0) = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) / det;
    IM(1, 0) = -(M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0)) / det;
    IM(2, 0) = (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0)) / det;
    IM(0, 1) = -(M(0, 1) * M(2, 2) - M(0, 2) * M(2, 1)) / det;
    IM(1, 1) = (M(0, 0) * M(2, 2) - M(0, 2) * M(2, 0)) / det;
    IM(2, 1) = -(M(0, 0) * M(2, 1) - M(0, 1) * M(2, 0)) / det;
    IM(0, 2) = (M(0, 1) * M(1, 2) - M(0, 2) * M(1, 1)) / det;
    IM(1, 2) = -(M(0, 0) * M(1, 2) - M(0, 2) * M(1, 0)) / det;
    IM(2, 2) = (M(0, 0) * M(1, 1) - M(0, 1) * M(1, 0)) / det;
#undef IM
#undef M
}

/* Math::invA for dim > 3 (linear_algebra.cpp:123-131, 167-175): identity,
 * then unpivoted Doolittle LU (KokkosBatched LU Unblocked) and SolveLU.
 * a[n][n] is overwritten by its LU factors. */
static void inv_lu(int n, double* a, double* ia)
{
    if (n == 1) { ia[0] = 1. / a[0]; return; }
    for (int i = 0; i < n * n; i++) ia[i] = 0.0;
    for (int i = 0; i < n; i++) ia[i * n + i] = 1.0;
    for (int k = 0; k < n; k++) {
        double piv = a[k * n + k];
        for (int i = k + 1; i < n; i++) a[i * n + k] /= piv;
        for (int i = k + 1; i < n; i++) {
            double lik = a[i * n + k];
            for (int j = k + 1; j < n; j++) a[i * n + j] -= lik * a[k * n + j];
        }
    }
    /* forward substitution with unit-lower L, then backward with U */
    for (int c = 0; c < n; c++) {
        for (int i = 0; i < n; i++) {
            double s = ia[i * n + c];
            for (int k = 0; k < i; k++) s -= a[i * n + k] * ia[k * n + c];
            ia[i * n + c] = s;
        }
        for (int i = n - 1; i >= 0; i--) {
            double s = ia[i * n + c];
            for (int k = i + 1; k < n; k++) s -= a[i * n + k] * ia[k * n + c];
            ia[i * n + c] = s / a[i * n + i];
        }
    }
}

void orc_inv_lu(int n, double* a, double* ia) { inv_lu(n, a, ia); }

/* ------------------------------------------------------------------------ */
/* the case                                                                  */
/* ------------------------------------------------------------------------ */

struct orc_case {
    int p, nb, ne, nnode, nif, flux_type;
    double gamma, R;
    double* coords; /* [nnode][3] */
    int* e2n;       /* [ne][8] */
    int* ifd;       /* [nif][6] */
    /* volume helpers at quadrature order p (helpers.cpp:5-51) */
    int nq;
    double *vq_pts, *vq_wts, *B, *Dref; /* B[nq][nb], Dref[nq][nb][3] */
    double *djac, *ijac;                 /* [ne][nq], [ne][nq][3][3] */
    double* vol;                         /* [ne] */
    double* iMM;                         /* [ne][nb][nb] (helpers.cpp:54-100) */
    /* face helpers (helpers.cpp:205-500) */
    int nqf;
    double* fwts;                 /* [nqf] */
    double* Bf;                   /* [6*nqf][nb] */
    int *qidxL, *qidxR;           /* [nif][nqf] */
    double* normals;              /* [nif][nqf][3] */
    /* IC / error quadrature at order 2*max(p,1) (base.cpp:114-223, post/main.cpp:59-99) */
    int nqe;
    double *eq_pts, *eq_wts, *Be, *ge_val, *ge_grad;
    int ic_type, ic_ndata;
    double ic_data[16];
    /* scratch */
    double *Uq, *vgUq, *Uqf, *UqL, *UqR, *Fq, *Fq_elem, *res;
    double *dU[4], *Uhold;
    long flux_fail;
};

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}
#define NT orc_get_threads()

int orc_nb(const orc_case* c) { return c->nb; }
int orc_nqf(const orc_case* c) { return c->nqf; }
double orc_total_volume(const orc_case* c)
{
    double v = 0.0;
    for (int e = 0; e < c->ne; e++) v += c->vol[e];
    return v;
}
long orc_flux_failures(const orc_case* c) { return c->flux_fail; }

/* geometric basis (LagrangeHex, gorder 1) values and gradients at pts */
static void gbasis_tables(int nq, const double* pts, double** gval, double** ggrad)
{
    *gval = malloc(sizeof(double) * nq * 8);
    *ggrad = malloc(sizeof(double) * nq * 8 * 3);
    orc_lagrange_hex_val(1, nq, pts, *gval);
    orc_lagrange_hex_grad(1, nq, pts, *ggrad);
}

/* BasisTools::get_element_jacobian, basis/tools.cpp:42-66:
 * jac(i,j) = sum_n X(n,i) * dphi_n/dxi_j  (Math::cATxB_to_C) */
static void elem_jac(const double* X /*[8][3]*/, const double* gg /*[8][3]*/, double* jac)
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0.0;
            for (int n = 0; n < 8; n++) s += X[n * 3 + i] * gg[n * 3 + j];
            jac[i * 3 + j] = s;
        }
}

static void elem_coords(const orc_case* c, int e, double* X)
{
    for (int n = 0; n < 8; n++)
        for (int d = 0; d < 3; d++) X[n * 3 + d] = c->coords[c->e2n[e * 8 + n] * 3 + d];
}

orc_case* orc_create(int p, int flux_type, double gamma, double gas_const,
                     int nnode, const double* coords, int nelem, const int* elem2node,
                     int nif, const int* ifdata)
{
    if (p < 0 || p > 8 || nelem <= 0 || nif < 0) return NULL;
    orc_case* c = calloc(1, sizeof(orc_case));
    c->p = p;
    c->nb = (p + 1) * (p + 1) * (p + 1);
    c->ne = nelem;
    c->nnode = nnode;
    c->nif = nif;
    c->flux_type = flux_type;
    c->gamma = gamma;
    c->R = gas_const;
    c->coords = malloc(sizeof(double) * nnode * 3);
    memcpy(c->coords, coords, sizeof(double) * nnode * 3);
    c->e2n = malloc(sizeof(int) * nelem * 8);
    memcpy(c->e2n, elem2node, sizeof(int) * nelem * 8);
    c->ifd = malloc(sizeof(int) * (nif > 0 ? nif : 1) * 6);
    if (nif > 0) memcpy(c->ifd, ifdata, sizeof(int) * nif * 6);
    const int nb = c->nb, ne = c->ne;

    /* --- inverse mass matrices, helpers.cpp:54-100 (quadrature order 2p) --- */
    {
        double *pts, *wts, *gv, *gg;
        int nqm = hex_quadrature(orc_hex_quadrature_order(2 * p), &pts, &wts);
        double* Bm = malloc(sizeof(double) * nqm * nb);
        orc_lagrange_hex_val(p, nqm, pts, Bm);
        gbasis_tables(nqm, pts, &gv, &gg);
        c->iMM = malloc(sizeof(double) * (size_t)ne * nb * nb);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (int e = 0; e < ne; e++) {
            double X[24], jac[9];
            double* S = malloc(sizeof(double) * nqm * nb);
            double* MM = malloc(sizeof(double) * nb * nb);
            elem_coords(c, e, X);
            for (int q = 0; q < nqm; q++) {
                elem_jac(X, gg + q * 24, jac);
                double cw = wts[q] * det3(jac);
                for (int j = 0; j < nb; j++) S[q * nb + j] = Bm[q * nb + j] * cw;
            }
            for (int i = 0; i < nb; i++)
                for (int j = 0; j < nb; j++) {
                    double s = 0.0;
                    for (int q = 0; q < nqm; q++) s += Bm[q * nb + i] * S[q * nb + j];
                    MM[i * nb + j] = s;
                }
            inv_lu(nb, MM, c->iMM + (size_t)e * nb * nb);
            free(S);
            free(MM);
        }
        free(pts); free(wts); free(Bm); free(gv); free(gg);
    }

    /* --- volume helpers, helpers.cpp:5-51 (quadrature order p) --- */
    {
        double *gv, *gg;
        c->nq = hex_quadrature(orc_hex_quadrature_order(p), &c->vq_pts, &c->vq_wts);
        const int nq = c->nq;
        c->B = malloc(sizeof(double) * nq * nb);
        c->Dref = malloc(sizeof(double) * nq * nb * 3);
        orc_lagrange_hex_val(p, nq, c->vq_pts, c->B);
        orc_lagrange_hex_grad(p, nq, c->vq_pts, c->Dref);
        gbasis_tables(nq, c->vq_pts, &gv, &gg);
        c->djac = malloc(sizeof(double) * (size_t)ne * nq);
        c->ijac = malloc(sizeof(double) * (size_t)ne * nq * 9);
        c->vol = malloc(sizeof(double) * ne);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (int e = 0; e < ne; e++) {
            double X[24], jac[9];
            elem_coords(c, e, X);
            double v = 0.0;
            for (int q = 0; q < nq; q++) {
                elem_jac(X, gg + q * 24, jac);
                double dj = det3(jac);
                c->djac[(size_t)e * nq + q] = dj;
                inv3(jac, c->ijac + ((size_t)e * nq + q) * 9);
            }
            /* MeshTools::get_element_volume, mesh/tools.cpp:28-36 */
            for (int q = 0; q < nq; q++) v += c->vq_wts[q] * c->djac[(size_t)e * nq + q];
            c->vol[e] = v;
        }
        free(gv); free(gg);
    }

    /* --- interior face helpers, helpers.cpp:205-500 --- */
    {
        double *fpts, *fw;
        c->nqf = quad_quadrature(orc_quad_quadrature_order(p), &fpts, &fw);
        const int nqf = c->nqf;
        c->fwts = fw;
        double* epts = malloc(sizeof(double) * 6 * nqf * 3);
        for (int f = 0; f < 6; f++) orc_points_on_face(f, 0, nqf, fpts, epts + f * nqf * 3);
        c->Bf = malloc(sizeof(double) * 6 * nqf * nb);
        orc_lagrange_hex_val(p, 6 * nqf, epts, c->Bf);
        /* precompute_facequadrature_lookup, helpers.cpp:326-378 */
        c->qidxL = malloc(sizeof(int) * (nif > 0 ? nif : 1) * nqf);
        c->qidxR = malloc(sizeof(int) * (nif > 0 ? nif : 1) * nqf);
        for (int f = 0; f < nif; f++) {
            orc_face_pts_order(c->ifd[f * 6 + 2], nqf, c->qidxL + f * nqf);
            orc_face_pts_order(c->ifd[f * 6 + 5], nqf, c->qidxR + f * nqf);
        }
        /* precompute_normals, helpers.cpp:380-500 with shape.cpp:482-532:
         * face geometric-basis gradients at face 0's points (first two
         * coordinates, basis.cpp:306-338), nodes from the left element. */
        double* ref2 = malloc(sizeof(double) * nqf * 2);
        for (int q = 0; q < nqf; q++) {
            ref2[q * 2 + 0] = epts[q * 3 + 0];
            ref2[q * 2 + 1] = epts[q * 3 + 1];
        }
        double* fgg = malloc(sizeof(double) * nqf * 4 * 2);
        lagrange_quad_grad(1, nqf, ref2, fgg);
        c->normals = malloc(sizeof(double) * (nif > 0 ? nif : 1) * nqf * 3);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (int f = 0; f < nif; f++) {
            int eL = c->ifd[f * 6 + 0], fL = c->ifd[f * 6 + 1];
            double X[24], FC[12];
            int lf[4];
            elem_coords(c, eL, X);
            orc_local_nodes_on_face(fL, 1, lf);
            for (int n = 0; n < 4; n++)
                for (int d = 0; d < 3; d++) FC[n * 3 + d] = X[lf[n] * 3 + d];
            for (int q = 0; q < nqf; q++) {
                double xg[3][2];
                for (int j = 0; j < 3; j++)
                    for (int d = 0; d < 2; d++) {
                        double s = 0.0;
                        for (int n = 0; n < 4; n++) s += FC[n * 3 + j] * fgg[(q * 4 + n) * 2 + d];
                        xg[j][d] = s;
                    }
                double a[3] = {xg[0][0], xg[1][0], xg[2][0]};
                double b[3] = {xg[0][1], xg[1][1], xg[2][1]};
                double* N = c->normals + ((size_t)f * nqf + q) * 3;
                /* Math::cross, linear_algebra.cpp:36-41; sign +1 (left rank) */
                N[0] = (a[1] * b[2] - a[2] * b[1]) * 1.0;
                N[1] = (a[2] * b[0] - a[0] * b[2]) * 1.0;
                N[2] = (a[0] * b[1] - a[1] * b[0]) * 1.0;
            }
        }
        free(fpts); free(epts); free(ref2); free(fgg);
    }

    /* --- IC / error quadrature, base.cpp:124-161 and post/main.cpp:59-99 --- */
    {
        int pp = p > 1 ? p : 1;
        c->nqe = hex_quadrature(orc_hex_quadrature_order(2 * pp), &c->eq_pts, &c->eq_wts);
        c->Be = malloc(sizeof(double) * c->nqe * nb);
        orc_lagrange_hex_val(p, c->nqe, c->eq_pts, c->Be);
        gbasis_tables(c->nqe, c->eq_pts, &c->ge_val, &c->ge_grad);
    }

    /* --- work arrays (base.cpp:427-432, 564-598; stepper.cpp:57-69) --- */
    size_t nstate = (size_t)ne * nb * NS;
    c->Uq = malloc(sizeof(double) * (size_t)ne * c->nq * NS);
    c->vgUq = malloc(sizeof(double) * (size_t)ne * c->nq * NS * 3);
    c->Uqf = malloc(sizeof(double) * (size_t)ne * 6 * c->nqf * NS);
    c->UqL = malloc(sizeof(double) * (size_t)(nif > 0 ? nif : 1) * c->nqf * NS);
    c->UqR = malloc(sizeof(double) * (size_t)(nif > 0 ? nif : 1) * c->nqf * NS);
    c->Fq = malloc(sizeof(double) * (size_t)(nif > 0 ? nif : 1) * c->nqf * NS);
    c->Fq_elem = calloc((size_t)ne * 6 * c->nqf * NS, sizeof(double));
    c->res = malloc(sizeof(double) * nstate);
    for (int s = 0; s < 4; s++) c->dU[s] = malloc(sizeof(double) * nstate);
    c->Uhold = malloc(sizeof(double) * nstate);
    return c;
}

void orc_destroy(orc_case* c)
{
    if (!c) return;
    free(c->coords); free(c->e2n); free(c->ifd);
    free(c->vq_pts); free(c->vq_wts); free(c->B); free(c->Dref);
    free(c->djac); free(c->ijac); free(c->vol); free(c->iMM);
    free(c->fwts); free(c->Bf); free(c->qidxL); free(c->qidxR); free(c->normals);
    free(c->eq_pts); free(c->eq_wts); free(c->Be); free(c->ge_val); free(c->ge_grad);
    free(c->Uq); free(c->vgUq); free(c->Uqf); free(c->UqL); free(c->UqR); free(c->Fq);
    free(c->Fq_elem); free(c->res);
    for (int s = 0; s < 4; s++) free(c->dU[s]);
    free(c->Uhold);
    free(c);
}

void orc_set_ic(orc_case* c, int ic_type, int ndata, const double* data)
{
    c->ic_type = ic_type;
    c->ic_ndata = ndata > 16 ? 16 : ndata;
    for (int i = 0; i < c->ic_ndata; i++) c->ic_data[i] = data[i];
}

/* Solver::init_state_from_fcn + SolverTools::L2_projection,
 * base.cpp:113-223, solver/tools.cpp:66-122 */
void orc_project_ic(orc_case* c, double t, double* Uc)
{
    const int nb = c->nb, nq = c->nqe;
#pragma omp parallel for num_threads(NT) schedule(static)
    for (int e = 0; e < c->ne; e++) {
        double X[24], jac[9];
        double* f = malloc(sizeof(double) * nq * NS);
        double* rhs = malloc(sizeof(double) * nb * NS);
        elem_coords(c, e, X);
        for (int q = 0; q < nq; q++) {
            double xp[3];
            /* MeshTools::ref_to_phys, mesh/tools.cpp:19-26 (gbasis_val * X) */
            for (int d = 0; d < 3; d++) {
                double s = 0.0;
                for (int n = 0; n < 8; n++) s += c->ge_val[q * 8 + n] * X[n * 3 + d];
                xp[d] = s;
            }
            orc_ic_eval(c->ic_type, c->ic_ndata, c->ic_data, c->gamma, c->R, xp, t, f + q * NS);
            elem_jac(X, c->ge_grad + q * 24, jac);
            double cw = c->eq_wts[q] * det3(jac);
            for (int s = 0; s < NS; s++) f[q * NS + s] = f[q * NS + s] * cw;
        }
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS; s++) {
                double acc = 0.0;
                for (int q = 0; q < nq; q++) acc += c->Be[q * nb + b] * f[q * NS + s];
                rhs[b * NS + s] = acc;
            }
        const double* iM = c->iMM + (size_t)e * nb * nb;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS; s++) {
                double acc = 0.0;
                for (int k = 0; k < nb; k++) acc += iM[b * nb + k] * rhs[k * NS + s];
                Uc[((size_t)e * nb + b) * NS + s] = acc;
            }
        free(f);
        free(rhs);
    }
}

/* Solver::get_residual, base.cpp:401-561 */
void orc_residual(orc_case* c, const double* Uc, double* res)
{
    const int nb = c->nb, nq = c->nq, nqf = c->nqf, ne = c->ne, nif = c->nif;
    const size_t nstate = (size_t)ne * nb * NS;
    long fails = 0;
    /* Math::fill(res, 0), base.cpp:404-406 */
#pragma omp parallel for num_threads(NT) schedule(static)
    for (long i = 0; i < (long)nstate; i++) res[i] = 0.0;

    /* get_element_residuals, base.cpp:415-468 */
#pragma omp parallel for num_threads(NT) schedule(static)
    for (int e = 0; e < ne; e++) {
        const double* U = Uc + (size_t)e * nb * NS;
        double* Uq = c->Uq + (size_t)e * nq * NS;
        double* vg = c->vgUq + (size_t)e * nq * NS * 3;
        /* evaluate_state: Uq_e = B * Uc_e, helpers.cpp:185-198 */
        for (int q = 0; q < nq; q++)
            for (int s = 0; s < NS; s++) {
                double acc = 0.0;
                for (int b = 0; b < nb; b++) acc += c->B[q * nb + b] * U[b * NS + s];
                Uq[q * NS + s] = acc;
            }
        /* VolumeFluxesFunctor, flux_functors_impl.h:46-115 */
        for (int q = 0; q < nq; q++) {
            double gF1[15], gF2[15];
            orc_conv_flux(c->gamma, Uq + q * NS, gF1);
            const double* ij = c->ijac + ((size_t)e * nq + q) * 9;
            const double dj = c->djac[(size_t)e * nq + q], w = c->vq_wts[q];
            for (int i = 0; i < 15; i++) gF2[i] = 0.;
            for (int d1 = 0; d1 < 3; d1++)
                for (int d2 = 0; d2 < 3; d2++)
                    for (int s = 0; s < NS; s++)
                        gF2[d1 * NS + s] += gF1[d2 * NS + s] * ij[d1 * 3 + d2] * dj * w;
            for (int d = 0; d < 3; d++)
                for (int s = 0; s < NS; s++) vg[(q * NS + s) * 3 + d] = gF2[d * NS + s];
        }
        /* calculate_volume_flux_integral, solver/tools.cpp:7-35 */
        double* r = res + (size_t)e * nb * NS;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS; s++)
                for (int q = 0; q < nq; q++)
                    for (int d = 0; d < 3; d++)
                        r[b * NS + s] += c->Dref[(q * nb + b) * 3 + d] * vg[(q * NS + s) * 3 + d];
        /* face traces: evaluate_state with the stacked face basis, base.cpp:504-507 */
        double* Uf = c->Uqf + (size_t)e * 6 * nqf * NS;
        for (int q = 0; q < 6 * nqf; q++)
            for (int s = 0; s < NS; s++) {
                double acc = 0.0;
                for (int b = 0; b < nb; b++) acc += c->Bf[q * nb + b] * U[b * NS + s];
                Uf[q * NS + s] = acc;
            }
    }

    /* construct_face_states (base.cpp:287-327) and the face flux functor
     * (flux_functors_impl.h:168-264); one rank, so no halo exchange */
#pragma omp parallel for num_threads(NT) schedule(static) reduction(+ : fails)
    for (int f = 0; f < nif; f++) {
        int eL = c->ifd[f * 6 + 0], fL = c->ifd[f * 6 + 1];
        int eR = c->ifd[f * 6 + 3], fR = c->ifd[f * 6 + 4];
        for (int q = 0; q < nqf; q++) {
            const double* UL = c->Uqf + (((size_t)eL * 6 + fL) * nqf + c->qidxL[f * nqf + q]) * NS;
            const double* UR = c->Uqf + (((size_t)eR * 6 + fR) * nqf + c->qidxR[f * nqf + q]) * NS;
            double* UqL = c->UqL + ((size_t)f * nqf + q) * NS;
            double* UqR = c->UqR + ((size_t)f * nqf + q) * NS;
            for (int s = 0; s < NS; s++) { UqL[s] = UL[s]; UqR[s] = UR[s]; }
            double F[NS];
            if (orc_num_flux(c->flux_type, c->gamma, UqL, UqR, c->normals + ((size_t)f * nqf + q) * 3, F))
                fails++;
            for (int s = 0; s < NS; s++) c->Fq[((size_t)f * nqf + q) * NS + s] = F[s] * c->fwts[q];
        }
    }
    c->flux_fail += fails;

    /* construct_flux_state, base.cpp:329-374 (serial: two faces of one
     * element write disjoint slots, but keep the reference's order) */
    for (int f = 0; f < nif; f++) {
        int eL = c->ifd[f * 6 + 0], fL = c->ifd[f * 6 + 1];
        int eR = c->ifd[f * 6 + 3], fR = c->ifd[f * 6 + 4];
        for (int q = 0; q < nqf; q++)
            for (int s = 0; s < NS; s++) {
                double v = c->Fq[((size_t)f * nqf + q) * NS + s];
                c->Fq_elem[(((size_t)eL * 6 + fL) * nqf + c->qidxL[f * nqf + q]) * NS + s] = -1.0 * v;
                c->Fq_elem[(((size_t)eR * 6 + fR) * nqf + c->qidxR[f * nqf + q]) * NS + s] = v;
            }
    }

    /* calculate_face_flux_integral: res_e += Bf^T * Fq_elem_e, tools.cpp:38-63 */
#pragma omp parallel for num_threads(NT) schedule(static)
    for (int e = 0; e < ne; e++) {
        const double* Fe = c->Fq_elem + (size_t)e * 6 * nqf * NS;
        double* r = res + (size_t)e * nb * NS;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS; s++) {
                double acc = 0.0;
                for (int q = 0; q < 6 * nqf; q++) acc += c->Bf[q * nb + b] * Fe[q * NS + s];
                r[b * NS + s] += acc;
            }
    }
}

/* SolverTools::mult_inv_mass_matrix, solver/tools.cpp:124-139:
 * dU_e = dt * iMM_e * res_e */
static void mult_inv_mass(orc_case* c, double dt, const double* res, double* dU)
{
    const int nb = c->nb;
#pragma omp parallel for num_threads(NT) schedule(static)
    for (int e = 0; e < c->ne; e++) {
        const double* iM = c->iMM + (size_t)e * nb * nb;
        const double* r = res + (size_t)e * nb * NS;
        double* d = dU + (size_t)e * nb * NS;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS; s++) {
                double acc = 0.0;
                for (int k = 0; k < nb; k++) acc += iM[b * nb + k] * r[k * NS + s];
                d[b * NS + s] = dt * acc;
            }
    }
}

/* RK4<3>::take_time_step, numerics/timestepping/stepper.cpp:71-142 */
void orc_rk4_steps(orc_case* c, double* Uc, double dt, int nsteps)
{
    const long n = (long)c->ne * c->nb * NS;
    double *d1 = c->dU[0], *d2 = c->dU[1], *d3 = c->dU[2], *d4 = c->dU[3], *Uh = c->Uhold;
    for (int it = 0; it < nsteps; it++) {
        memcpy(Uh, Uc, sizeof(double) * n);
        orc_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d1);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (long i = 0; i < n; i++) Uc[i] = 0.5 * d1[i] + 1.0 * Uh[i];
        orc_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d2);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (long i = 0; i < n; i++) Uc[i] = 0.5 * d2[i] + 1.0 * Uh[i];
        orc_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d3);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (long i = 0; i < n; i++) Uc[i] = 1.0 * d3[i] + 1.0 * Uh[i];
        orc_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d4);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (long i = 0; i < n; i++) {
            double a = d4[i] + 2.0 * d3[i];
            a = a + 2.0 * d2[i];
            a = a + 1.0 * d1[i];
            Uh[i] = Uh[i] + (1.0 / 6.0) * a;
            Uc[i] = Uh[i];
        }
    }
}

/* FE<3>::take_time_step, stepper.cpp:23-55 */
void orc_fe_steps(orc_case* c, double* Uc, double dt, int nsteps)
{
    const long n = (long)c->ne * c->nb * NS;
    for (int it = 0; it < nsteps; it++) {
        orc_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, c->dU[0]);
#pragma omp parallel for num_threads(NT) schedule(static)
        for (long i = 0; i < n; i++) Uc[i] = Uc[i] + 1.0 * c->dU[0][i];
    }
}

/* get_error with ord = 2 and volume normalisation, post/main.cpp:30-201 */
void orc_l2_error(orc_case* c, const double* Uc, double t, double* err)
{
    const int nb = c->nb, nq = c->nqe;
    double tot[NS] = {0, 0, 0, 0, 0};
    double* per = malloc(sizeof(double) * c->ne * NS);
#pragma omp parallel for num_threads(NT) schedule(static)
    for (int e = 0; e < c->ne; e++) {
        double X[24], jac[9], Ue[NS], Uq[NS], xp[3];
        double acc[NS] = {0, 0, 0, 0, 0};
        elem_coords(c, e, X);
        const double* U = Uc + (size_t)e * nb * NS;
        for (int q = 0; q < nq; q++) {
            for (int s = 0; s < NS; s++) {
                double a = 0.0;
                for (int b = 0; b < nb; b++) a += c->Be[q * nb + b] * U[b * NS + s];
                Uq[s] = a;
            }
            for (int d = 0; d < 3; d++) {
                double s = 0.0;
                for (int n = 0; n < 8; n++) s += c->ge_val[q * 8 + n] * X[n * 3 + d];
                xp[d] = s;
            }
            orc_ic_eval(c->ic_type, c->ic_ndata, c->ic_data, c->gamma, c->R, xp, t, Ue);
            elem_jac(X, c->ge_grad + q * 24, jac);
            double dj = det3(jac);
            for (int s = 0; s < NS; s++) {
                double d = Uq[s] - Ue[s];
                acc[s] += d * d * c->eq_wts[q] * dj;
            }
        }
        for (int s = 0; s < NS; s++) per[e * NS + s] = acc[s];
    }
    for (int e = 0; e < c->ne; e++)
        for (int s = 0; s < NS; s++) tot[s] += per[e * NS + s];
    free(per);
    double V = orc_total_volume(c);
    for (int s = 0; s < NS; s++) err[s] = sqrt(tot[s] / V);
}

void orc_face_normals(const orc_case* c, double* N)
{
    memcpy(N, c->normals, sizeof(double) * (size_t)c->nif * c->nqf * 3);
}

void orc_face_quad_idx(const orc_case* c, int* idxL, int* idxR)
{
    memcpy(idxL, c->qidxL, sizeof(int) * (size_t)c->nif * c->nqf);
    memcpy(idxR, c->qidxR, sizeof(int) * (size_t)c->nif * c->nqf);
}

/* physical coordinates of an element's face quadrature points (orientation 0) */
void orc_face_points_phys(const orc_case* c, int elem, int face, double* Xout)
{
    double *fpts, *fw, X[24];
    int nqf = quad_quadrature(orc_quad_quadrature_order(c->p), &fpts, &fw);
    double* ep = malloc(sizeof(double) * nqf * 3);
    double* gv = malloc(sizeof(double) * nqf * 8);
    orc_points_on_face(face, 0, nqf, fpts, ep);
    orc_lagrange_hex_val(1, nqf, ep, gv);
    elem_coords(c, elem, X);
    for (int q = 0; q < nqf; q++)
        for (int d = 0; d < 3; d++) {
            double s = 0.0;
            for (int n = 0; n < 8; n++) s += gv[q * 8 + n] * X[n * 3 + d];
            Xout[q * 3 + d] = s;
        }
    free(fpts); free(fw); free(ep); free(gv);
}
