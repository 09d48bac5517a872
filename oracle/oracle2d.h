/*
 * oracle2d.h -- CPU restatement of DG-MPI's 2D Euler residual + RK path on
 * quadrilateral meshes (oracle2d.c).  TEST INFRASTRUCTURE ONLY: the product
 * path never links, loads or calls it.
 *
 * Pinned against the reference's 2D convergence table
 * (examples/isentropic_vortex/convergence.py: HLLC, LagrangeQuad, RK4,
 * dt = 1e-3 to t = 1, periodic boxes of N x N quadrilaterals).
 * State layout Uc[ne][nb][4], row-major; nb = (p+1)^2.
 */
#ifndef DG_ORACLE2D_H
#define DG_ORACLE2D_H

#ifdef __cplusplus
extern "C" {
#endif

/* the reference's 2D isentropic vortex (physics/euler/functions.cpp:94-145):
 * data = {rho, u, v, p, vortex strength}, centred at the origin at t = 0,
 * advected with (u, v), not wrapped; the other ORC_IC_* codes evaluate the 3D
 * families at (x, y, 0) (ORC_IC_UNIFORM: data = the four conserved values) */
#define ORC2_IC_VORTEX 5

typedef struct orc2_case orc2_case;

/* coords[nnode][2]; elem2node[nelem][4] (gbasis order, x fastest);
 * ifdata[nif][6] = (elemL, faceL, orientL, elemR, faceR, orientR) as the
 * mesh file's IFaceData.  Returns NULL on error. */
orc2_case* orc2_create(int p, int flux_type, double gamma, double gas_const, int nnode, const double* coords,
                       int nelem, const int* elem2node, int nif, const int* ifdata);
void orc2_destroy(orc2_case* c);
int orc2_nb(const orc2_case* c);
int orc2_nqf(const orc2_case* c);
void orc2_set_ic(orc2_case* c, int ic_type, int ndata, const double* data);
void orc2_project_ic(orc2_case* c, double t, double* Uc);
void orc2_residual(orc2_case* c, const double* Uc, double* res);
void orc2_rk4_steps(orc2_case* c, double* Uc, double dt, int nsteps);
void orc2_fe_steps(orc2_case* c, double* Uc, double dt, int nsteps);
void orc2_l2_error(orc2_case* c, const double* Uc, double t, double* err /*[4]*/);
double orc2_total_volume(const orc2_case* c);
long orc2_flux_failures(const orc2_case* c);
void orc2_face_normals(const orc2_case* c, double* N /*[nif][nqf][2]*/);
void orc2_points_on_face(int face, int orient, int np, const double* s, double* epts);
void orc2_face_pts_order(int orient, int npts, int* order);

#ifdef __cplusplus
}
#endif
#endif
