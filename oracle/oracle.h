/*
 * oracle.h -- CPU restatement of DG-MPI's 3D Euler residual + RK hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark may
 * load it, and only as the checker.  The product path (libdg_b200.so) never
 * links, loads or calls it.
 *
 * It restates the reference's *dense per-element* algorithm (the Kokkos
 * build of IhmeGroup/DG-MPI): per-element B*U GEMMs, per-quadrature-point
 * geometry (jac/djac/ijac), per-element dense inverse mass matrices obtained
 * by an unpivoted LU, face states gathered through the quad_idx_L/R
 * permutations, Lax-Friedrichs / HLLC numerical fluxes, the L=-F / R=+F
 * scatter, the face lift Bf^T * Fq_elem, and the stored-stage RK4.  Every
 * function cites the reference file:line it follows (paths relative to the
 * reference project root).
 *
 * Parity pins: the end-to-end 3D isentropic-vortex regression
 * (examples/euler/3D/isentropic_vortex/regression_data.txt:13-17), the
 * basis/quadrature/nodes unit tests (test/numerics/...), and the reference's
 * own Gauss-Legendre tables (src/numerics/nodes.cpp, quadrature/segment.cpp).
 *
 * State layout everywhere: Uc[ne][nb][5], row-major (Kokkos LayoutRight, the
 * CPU build's layout, src/io/writer.cpp:72 "Stored Layout" = true).
 */
#ifndef DG_ORACLE_H
#define DG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NS 5

enum { ORC_FLUX_LF = 0, ORC_FLUX_HLLC = 1 };

/* Initial-condition / exact-solution families.
 *   UNIFORM     : data[0..4] = conserved state (physics/base/base.cpp:150-158)
 *   VORTEX_REF  : the reference's hard-coded 3D vortex (x-z plane, Mach 1,
 *                 radius 0.1, centre (0.5, *, 0.5)), ignores data and t
 *                 (physics/euler/functions.cpp:147-191)
 *   SPHERE      : smooth sphere (physics/base/base.cpp:177-194)
 *   VORTEX_XY   : the 2D isentropic vortex of physics/euler/functions.cpp:94-145
 *                 extruded in z, centred at (xc, yc), advected with (u, v),
 *                 periodic in x/y with periods (Lx, Ly):
 *                 data = {rho, u, v, p, beta, xc, yc, Lx, Ly}; gas constant 1
 *   TAYLOR_GREEN: rho=1, u=(sin x cos y cos z, -cos x sin y cos z, 0),
 *                 p = 1/(gamma M^2) + (cos2x+cos2y)(cos2z+2)/16; data = {M}
 */
enum {
    ORC_IC_UNIFORM = 0,
    ORC_IC_VORTEX_REF = 1,
    ORC_IC_SPHERE = 2,
    ORC_IC_VORTEX_XY = 3,
    ORC_IC_TAYLOR_GREEN = 4
};

/* ---- quadrature / basis primitives (for the golden-vector tests) ---- */
int  orc_hex_quadrature_order(int order);           /* quadrature/tools.cpp:7-17 */
int  orc_quad_quadrature_order(int order);          /* quadrature/quadrilateral.cpp:36-41 */
int  orc_segment_quadrature_order(int order);       /* quadrature/segment.cpp:424-426 */
int  orc_num_quadrature_points_1d(int qorder);      /* quadrature/tools.cpp:20-24 */
void orc_gauss_legendre_1d(int qorder, double* pts, double* wts);
void orc_equidistant_nodes(double start, double stop, int n, double* x);
void orc_lagrange_1d_val(double x, int nn, const double* xn, double* phi);
void orc_lagrange_1d_grad(double x, int nn, const double* xn, double* gphi);
void orc_lagrange_hex_val(int p, int nq, const double* xq, double* val);
void orc_lagrange_hex_grad(int p, int nq, const double* xq, double* grad);
void orc_face_pts_order(int orient, int npts, int* order);
void orc_points_on_face(int face, int orient, int np, const double* fpts, double* epts);
void orc_local_nodes_on_face(int face, int gorder, int* lfnodes);
/* Math::invA for n > 3 (linear_algebra.cpp:123-131): unpivoted LU inverse;
 * a[n][n] is overwritten */
void orc_inv_lu(int n, double* a, double* ia);

/* ---- pointwise physics ---- */
double orc_pressure(double gamma, const double* U);
double orc_maxwavespeed(double gamma, const double* U);
void   orc_conv_flux(double gamma, const double* U, double* Fdir /*[15]*/);
/* returns 0, or -1 when HLLC finds no valid wave ordering (the reference asserts) */
int    orc_num_flux(int flux_type, double gamma, const double* UL, const double* UR,
                    const double* N, double* F);
void   orc_ic_eval(int ic_type, int ndata, const double* data, double gamma,
                   double R, const double* x, double t, double* U);

/* ---- a full case on a hex mesh given in the reference's mesh-file form ---- */
typedef struct orc_case orc_case;

/* coords[nnode][3]; elem2node[nelem][8] (gbasis order, x fastest);
 * ifdata[nif][6] = (elemL, faceL, orientL, elemR, faceR, orientR) exactly as
 * the HDF5 IFaceData dataset (mesh/mesh.cpp:144-160). Returns NULL on error. */
orc_case* orc_create(int p, int flux_type, double gamma, double gas_const,
                     int nnode, const double* coords,
                     int nelem, const int* elem2node,
                     int nif, const int* ifdata);
void orc_destroy(orc_case* c);
int  orc_nb(const orc_case* c);
int  orc_nqf(const orc_case* c);
void orc_set_ic(orc_case* c, int ic_type, int ndata, const double* data);
void orc_project_ic(orc_case* c, double t, double* Uc);
void orc_residual(orc_case* c, const double* Uc, double* res);
void orc_rk4_steps(orc_case* c, double* Uc, double dt, int nsteps);
void orc_fe_steps(orc_case* c, double* Uc, double dt, int nsteps);
void orc_l2_error(orc_case* c, const double* Uc, double t, double* err);
double orc_total_volume(const orc_case* c);
/* interior-face tables, for tests of the mesh generator */
void orc_face_normals(const orc_case* c, double* N /*[nif][nqf][3]*/);
void orc_face_quad_idx(const orc_case* c, int* idxL, int* idxR /*[nif][nqf]*/);
void orc_face_points_phys(const orc_case* c, int elem, int face, double* X /*[nqf][3]*/);
/* number of HLLC calls that hit the reference's assert branch so far */
long orc_flux_failures(const orc_case* c);

void orc_set_threads(int n);
int  orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
