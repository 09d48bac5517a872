/*
 * oracle2d.c -- CPU restatement of DG-MPI's 2D Euler residual + RK path on
 * quadrilateral meshes (Solver<2> with LagrangeQuad), the dense per-element
 * algorithm of the Kokkos build.
 *
 * TEST INFRASTRUCTURE ONLY, like oracle.c: only the tests, the smoke check
 * and the benchmark's CPU legs load it, and only as the checker.
 *
 * It follows the same reference code as the 3D oracle with the quadrilateral
 * branches of the shape / quadrature functions:
 *   - LagrangeQuad basis, node index j(p+1)+i, x fastest
 *     (basis/tools.cpp:151-213);
 *   - volume quadrature of order 2p+3 with (p+2)^2 Gauss points, j-major
 *     (quadrature/quadrilateral.cpp:7-41, helpers.cpp:123); the mass matrix
 *     on order 4p+3 ((2p+2)^2 points, base.cpp:78); IC projection and post
 *     error on order 4 max(p,1)+3 (base.cpp:124-161, post/main.cpp:59-99);
 *   - faces are segments: Gauss-Legendre of order 2p+1, p+1 points
 *     (quadrature/segment.cpp:424-426, helpers.cpp:225), mapped onto each
 *     face between its two corner nodes (get_points_on_face_quadrilateral,
 *     shape.cpp:69-122), point orders for the two orientations
 *     (shape.cpp:43-66);
 *   - face normals from the left element's face nodes
 *     (get_local_nodes_on_face_quadrilateral, shape.cpp:125-152) and the
 *     LagrangeSeg p=1 gradient: N = (dy/ds, -dx/ds) (shape.cpp:154-210,
 *     helpers.cpp:380-500);
 *   - the pointwise physics is the 3D oracle's on embedded states
 *     (rho, rho u, rho v, 0, rho E) and normals (nx, ny, 0): the reference's
 *     2D flux, pressure, Lax-Friedrichs and HLLC (functions.cpp:43-61,
 *     196-297) are the 3D ones with the third components left out, and the
 *     zero terms change no rounding.
 * State layout: Uc[ne][nb][4], row-major.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"
#include "oracle2d.h"

#define NS2 4

struct orc2_case {
    int p, nb, ne, nnode, nif, flux_type;
    double gamma, R;
    double* coords; /* [nnode][2] */
    int* e2n;       /* [ne][4] */
    int* ifd;       /* [nif][6] */
    /* volume */
    int nq;
    double *vq_wts, *B, *Dref; /* B[nq][nb], Dref[nq][nb][2] */
    double *djac, *ijac, *vol; /* per element and point */
    double* iMM;               /* [ne][nb][nb] */
    /* faces */
    int nqf;
    double *fwts, *Bf;     /* Bf[4 * nqf][nb] */
    int *qidxL, *qidxR;    /* [nif][nqf] */
    double* normals;       /* [nif][nqf][2] */
    /* IC / error */
    int nqe;
    double *eq_wts, *Be, *ge_val, *ge_grad;
    int ic_type, ic_ndata;
    double ic_data[16];
    /* work */
    double *Uq, *vgUq, *Uqf, *Fq, *Fq_elem, *res, *dU[4], *Uhold;
    long flux_fail;
};

static int nthreads(void) { return orc_get_threads(); }

/* QuadrilateralQuadrature::get_quadrature_gauss_legendre, quadrilateral.cpp:7-34 */
static int quad_rule(int qorder, double** pts, double** wts)
{
    int n = orc_num_quadrature_points_1d(qorder);
    double* x = malloc(sizeof(double) * n);
    double* w = malloc(sizeof(double) * n);
    orc_gauss_legendre_1d(qorder, x, w);
    *pts = malloc(sizeof(double) * n * n * 2);
    *wts = malloc(sizeof(double) * n * n);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            (*pts)[(j * n + i) * 2 + 0] = x[i];
            (*pts)[(j * n + i) * 2 + 1] = x[j];
            (*wts)[j * n + i] = w[i] * w[j];
        }
    free(x);
    free(w);
    return n * n;
}

/* get_lagrange_basis_val_2D / _grad_2D, basis/tools.cpp:151-213 */
static void quad_val(int p, int nq, const double* xq, double* val)
{
    int n = p + 1;
    double xn[16], vx[16], vy[16];
    orc_equidistant_nodes(-1.0, 1.0, n, xn);
    for (int q = 0; q < nq; q++) {
        orc_lagrange_1d_val(xq[q * 2 + 0], n, xn, vx);
        orc_lagrange_1d_val(xq[q * 2 + 1], n, xn, vy);
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) val[q * n * n + j * n + i] = vx[i] * vy[j];
    }
}

static void quad_grad(int p, int nq, const double* xq, double* grad)
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

/* corner nodes of a face in traversal order (get_points_on_face_quadrilateral,
 * shape.cpp:69-122; the same lists as get_local_nodes_on_face_quadrilateral at
 * gorder 1, shape.cpp:125-152) */
static const int kFaceNodes[4][2] = {{0, 1}, {1, 3}, {3, 2}, {2, 0}};

void orc2_points_on_face(int face, int orient, int np, const double* s, double* epts)
{
    static const double xr[4] = {-1., 1., -1., 1.}, yr[4] = {-1., -1., 1., 1.};
    int a = kFaceNodes[face][0], b = kFaceNodes[face][1];
    if (orient == 1) {
        int t = a;
        a = b;
        b = t;
    }
    for (int i = 0; i < np; i++) {
        double b1 = (s[i] + 1.) / 2., b0 = 1.0 - b1;
        epts[i * 2 + 0] = b0 * xr[a] + b1 * xr[b];
        epts[i * 2 + 1] = b0 * yr[a] + b1 * yr[b];
    }
}

/* get_face_pts_order_wrt_orient0_quadrilateral, shape.cpp:43-66 */
void orc2_face_pts_order(int orient, int npts, int* order)
{
    for (int i = 0; i < npts; i++) order[i] = orient == 1 ? npts - 1 - i : i;
}

static void elem_coords(const orc2_case* c, int e, double* X)
{
    for (int n = 0; n < 4; n++)
        for (int d = 0; d < 2; d++) X[n * 2 + d] = c->coords[c->e2n[e * 4 + n] * 2 + d];
}

/* get_element_jacobian (basis/tools.cpp:42-66) for dim 2: jac(i,j) = sum_n X(n,i) dphi_n/dxi_j */
static void elem_jac(const double* X, const double* gg /*[4][2]*/, double* jac)
{
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            double s = 0.0;
            for (int n = 0; n < 4; n++) s += X[n * 2 + i] * gg[n * 2 + j];
            jac[i * 2 + j] = s;
        }
}

/* Math::det and Math::invA for dim 2 (linear_algebra.cpp:99-107, 244-253) */
static double det2(const double* m) { return m[0] * m[3] - m[1] * m[2]; }

static void inv2(const double* m, double* im)
{
    double d = m[0] * m[3] - m[1] * m[2];
    im[0] = m[3] / d;
    im[1] = -m[1] / d;
    im[2] = -m[2] / d;
    im[3] = m[0] / d;
}

static void embed(const double* U4, double* U5)
{
    U5[0] = U4[0];
    U5[1] = U4[1];
    U5[2] = U4[2];
    U5[3] = 0.0;
    U5[4] = U4[3];
}

/* the state of a 2D IC / exact solution at (x, y): the 3D families at
 * (x, y, 0) without their third momentum; ORC2_IC_VORTEX is the reference's
 * 2D isentropic vortex (functions.cpp:94-145), centred at the origin and not
 * wrapped: the x-y family with centre (0, 0) and no period */
static void ic2(const orc2_case* c, const double* x2, double t, double* U4)
{
    double x3[3] = {x2[0], x2[1], 0.0}, U5[5];
    if (c->ic_type == ORC2_IC_VORTEX) {
        double d[9] = {0, 0, 0, 0, 0, 0.0, 0.0, 1e300, 1e300};
        for (int i = 0; i < 5 && i < c->ic_ndata; i++) d[i] = c->ic_data[i];
        orc_ic_eval(ORC_IC_VORTEX_XY, 9, d, c->gamma, c->R, x3, t, U5);
    } else if (c->ic_type == ORC_IC_UNIFORM) {
        double d[5] = {0, 0, 0, 0, 0};
        d[0] = c->ic_data[0];
        d[1] = c->ic_data[1];
        d[2] = c->ic_data[2];
        d[4] = c->ic_data[3];
        orc_ic_eval(ORC_IC_UNIFORM, 5, d, c->gamma, c->R, x3, t, U5);
    } else {
        orc_ic_eval(c->ic_type, c->ic_ndata, c->ic_data, c->gamma, c->R, x3, t, U5);
    }
    U4[0] = U5[0];
    U4[1] = U5[1];
    U4[2] = U5[2];
    U4[3] = U5[4];
}

int orc2_nb(const orc2_case* c) { return c->nb; }
int orc2_nqf(const orc2_case* c) { return c->nqf; }
long orc2_flux_failures(const orc2_case* c) { return c->flux_fail; }
double orc2_total_volume(const orc2_case* c)
{
    double v = 0.0;
    for (int e = 0; e < c->ne; e++) v += c->vol[e];
    return v;
}

orc2_case* orc2_create(int p, int flux_type, double gamma, double gas_const, int nnode, const double* coords,
                       int nelem, const int* elem2node, int nif, const int* ifdata)
{
    if (p < 0 || p > 8 || nelem <= 0 || nif < 0) return NULL;
    orc2_case* c = calloc(1, sizeof(orc2_case));
    c->p = p;
    c->nb = (p + 1) * (p + 1);
    c->ne = nelem;
    c->nnode = nnode;
    c->nif = nif;
    c->flux_type = flux_type;
    c->gamma = gamma;
    c->R = gas_const;
    c->coords = malloc(sizeof(double) * nnode * 2);
    memcpy(c->coords, coords, sizeof(double) * nnode * 2);
    c->e2n = malloc(sizeof(int) * nelem * 4);
    memcpy(c->e2n, elem2node, sizeof(int) * nelem * 4);
    c->ifd = malloc(sizeof(int) * (nif > 0 ? nif : 1) * 6);
    if (nif > 0) memcpy(c->ifd, ifdata, sizeof(int) * nif * 6);
    const int nb = c->nb, ne = c->ne;

    /* inverse mass matrices, helpers.cpp:54-100, quadrature order for 2p */
    {
        double *pts, *wts;
        int nqm = quad_rule(orc_quad_quadrature_order(2 * p), &pts, &wts);
        double* Bm = malloc(sizeof(double) * nqm * nb);
        double* gg = malloc(sizeof(double) * nqm * 4 * 2);
        quad_val(p, nqm, pts, Bm);
        quad_grad(1, nqm, pts, gg);
        c->iMM = malloc(sizeof(double) * (size_t)ne * nb * nb);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int e = 0; e < ne; e++) {
            double X[8], jac[4];
            double* S = malloc(sizeof(double) * nqm * nb);
            double* MM = malloc(sizeof(double) * nb * nb);
            elem_coords(c, e, X);
            for (int q = 0; q < nqm; q++) {
                elem_jac(X, gg + q * 8, jac);
                double cw = wts[q] * det2(jac);
                for (int j = 0; j < nb; j++) S[q * nb + j] = Bm[q * nb + j] * cw;
            }
            for (int i = 0; i < nb; i++)
                for (int j = 0; j < nb; j++) {
                    double s = 0.0;
                    for (int q = 0; q < nqm; q++) s += Bm[q * nb + i] * S[q * nb + j];
                    MM[i * nb + j] = s;
                }
            orc_inv_lu(nb, MM, c->iMM + (size_t)e * nb * nb);
            free(S);
            free(MM);
        }
        free(pts); free(wts); free(Bm); free(gg);
    }

    /* volume helpers, helpers.cpp:5-51 */
    {
        double* pts;
        c->nq = quad_rule(orc_quad_quadrature_order(p), &pts, &c->vq_wts);
        const int nq = c->nq;
        c->B = malloc(sizeof(double) * nq * nb);
        c->Dref = malloc(sizeof(double) * nq * nb * 2);
        double* gg = malloc(sizeof(double) * nq * 4 * 2);
        quad_val(p, nq, pts, c->B);
        quad_grad(p, nq, pts, c->Dref);
        quad_grad(1, nq, pts, gg);
        c->djac = malloc(sizeof(double) * (size_t)ne * nq);
        c->ijac = malloc(sizeof(double) * (size_t)ne * nq * 4);
        c->vol = malloc(sizeof(double) * ne);
        for (int e = 0; e < ne; e++) {
            double X[8], jac[4], v = 0.0;
            elem_coords(c, e, X);
            for (int q = 0; q < nq; q++) {
                elem_jac(X, gg + q * 8, jac);
                c->djac[(size_t)e * nq + q] = det2(jac);
                inv2(jac, c->ijac + ((size_t)e * nq + q) * 4);
            }
            for (int q = 0; q < nq; q++) v += c->vq_wts[q] * c->djac[(size_t)e * nq + q];
            c->vol[e] = v;
        }
        free(pts);
        free(gg);
    }

    /* interior faces: segment quadrature, face basis, lookups and normals */
    {
        int qo = orc_segment_quadrature_order(p);
        int nqf = orc_num_quadrature_points_1d(qo);
        c->nqf = nqf;
        double* s = malloc(sizeof(double) * nqf);
        c->fwts = malloc(sizeof(double) * nqf);
        orc_gauss_legendre_1d(qo, s, c->fwts);
        double* epts = malloc(sizeof(double) * 4 * nqf * 2);
        for (int f = 0; f < 4; f++) orc2_points_on_face(f, 0, nqf, s, epts + f * nqf * 2);
        c->Bf = malloc(sizeof(double) * 4 * nqf * nb);
        quad_val(p, 4 * nqf, epts, c->Bf);
        c->qidxL = malloc(sizeof(int) * (nif > 0 ? nif : 1) * nqf);
        c->qidxR = malloc(sizeof(int) * (nif > 0 ? nif : 1) * nqf);
        for (int f = 0; f < nif; f++) {
            orc2_face_pts_order(c->ifd[f * 6 + 2], nqf, c->qidxL + f * nqf);
            orc2_face_pts_order(c->ifd[f * 6 + 5], nqf, c->qidxR + f * nqf);
        }
        /* LagrangeSeg p = 1 gradient at face 0's x-coordinates: (-1/2, 1/2) */
        double xn[2], g[2];
        orc_equidistant_nodes(-1.0, 1.0, 2, xn);
        c->normals = malloc(sizeof(double) * (nif > 0 ? nif : 1) * nqf * 2);
        for (int f = 0; f < nif; f++) {
            int eL = c->ifd[f * 6 + 0], fL = c->ifd[f * 6 + 1];
            double X[8];
            elem_coords(c, eL, X);
            const int* ln = kFaceNodes[fL];
            for (int q = 0; q < nqf; q++) {
                orc_lagrange_1d_grad(epts[q * 2 + 0], 2, xn, g);
                double dx = X[ln[0] * 2 + 0] * g[0] + X[ln[1] * 2 + 0] * g[1];
                double dy = X[ln[0] * 2 + 1] * g[0] + X[ln[1] * 2 + 1] * g[1];
                c->normals[((size_t)f * nqf + q) * 2 + 0] = 1.0 * dy;
                c->normals[((size_t)f * nqf + q) * 2 + 1] = -1.0 * 1.0 * dx;
            }
        }
        free(s);
        free(epts);
    }

    /* IC / error quadrature */
    {
        int pp = p > 1 ? p : 1;
        double* pts;
        c->nqe = quad_rule(orc_quad_quadrature_order(2 * pp), &pts, &c->eq_wts);
        c->Be = malloc(sizeof(double) * c->nqe * nb);
        c->ge_val = malloc(sizeof(double) * c->nqe * 4);
        c->ge_grad = malloc(sizeof(double) * c->nqe * 4 * 2);
        quad_val(p, c->nqe, pts, c->Be);
        quad_val(1, c->nqe, pts, c->ge_val);
        quad_grad(1, c->nqe, pts, c->ge_grad);
        free(pts);
    }

    size_t nstate = (size_t)ne * nb * NS2;
    c->Uq = malloc(sizeof(double) * (size_t)ne * c->nq * NS2);
    c->vgUq = malloc(sizeof(double) * (size_t)ne * c->nq * NS2 * 2);
    c->Uqf = malloc(sizeof(double) * (size_t)ne * 4 * c->nqf * NS2);
    c->Fq = malloc(sizeof(double) * (size_t)(nif > 0 ? nif : 1) * c->nqf * NS2);
    c->Fq_elem = calloc((size_t)ne * 4 * c->nqf * NS2, sizeof(double));
    c->res = malloc(sizeof(double) * nstate);
    for (int k = 0; k < 4; k++) c->dU[k] = malloc(sizeof(double) * nstate);
    c->Uhold = malloc(sizeof(double) * nstate);
    return c;
}

void orc2_destroy(orc2_case* c)
{
    if (!c) return;
    free(c->coords); free(c->e2n); free(c->ifd);
    free(c->vq_wts); free(c->B); free(c->Dref); free(c->djac); free(c->ijac); free(c->vol); free(c->iMM);
    free(c->fwts); free(c->Bf); free(c->qidxL); free(c->qidxR); free(c->normals);
    free(c->eq_wts); free(c->Be); free(c->ge_val); free(c->ge_grad);
    free(c->Uq); free(c->vgUq); free(c->Uqf); free(c->Fq); free(c->Fq_elem); free(c->res);
    for (int k = 0; k < 4; k++) free(c->dU[k]);
    free(c->Uhold);
    free(c);
}

void orc2_set_ic(orc2_case* c, int ic_type, int ndata, const double* data)
{
    c->ic_type = ic_type;
    c->ic_ndata = ndata > 16 ? 16 : ndata;
    for (int i = 0; i < c->ic_ndata; i++) c->ic_data[i] = data[i];
}

/* Solver::init_state_from_fcn + L2 projection, base.cpp:113-223 */
void orc2_project_ic(orc2_case* c, double t, double* Uc)
{
    const int nb = c->nb, nq = c->nqe;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int e = 0; e < c->ne; e++) {
        double X[8], jac[4];
        double* f = malloc(sizeof(double) * nq * NS2);
        double* rhs = malloc(sizeof(double) * nb * NS2);
        elem_coords(c, e, X);
        for (int q = 0; q < nq; q++) {
            double xp[2];
            for (int d = 0; d < 2; d++) {
                double s = 0.0;
                for (int n = 0; n < 4; n++) s += c->ge_val[q * 4 + n] * X[n * 2 + d];
                xp[d] = s;
            }
            ic2(c, xp, t, f + q * NS2);
            elem_jac(X, c->ge_grad + q * 8, jac);
            double cw = c->eq_wts[q] * det2(jac);
            for (int s = 0; s < NS2; s++) f[q * NS2 + s] = f[q * NS2 + s] * cw;
        }
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS2; s++) {
                double acc = 0.0;
                for (int q = 0; q < nq; q++) acc += c->Be[q * nb + b] * f[q * NS2 + s];
                rhs[b * NS2 + s] = acc;
            }
        const double* iM = c->iMM + (size_t)e * nb * nb;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS2; s++) {
                double acc = 0.0;
                for (int k = 0; k < nb; k++) acc += iM[b * nb + k] * rhs[k * NS2 + s];
                Uc[((size_t)e * nb + b) * NS2 + s] = acc;
            }
        free(f);
        free(rhs);
    }
}

/* Solver<2>::get_residual, base.cpp:401-561 */
void orc2_residual(orc2_case* c, const double* Uc, double* res)
{
    const int nb = c->nb, nq = c->nq, nqf = c->nqf, ne = c->ne, nif = c->nif;
    long fails = 0;
    memset(res, 0, sizeof(double) * (size_t)ne * nb * NS2);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int e = 0; e < ne; e++) {
        const double* U = Uc + (size_t)e * nb * NS2;
        double* Uq = c->Uq + (size_t)e * nq * NS2;
        double* vg = c->vgUq + (size_t)e * nq * NS2 * 2;
        for (int q = 0; q < nq; q++)
            for (int s = 0; s < NS2; s++) {
                double acc = 0.0;
                for (int b = 0; b < nb; b++) acc += c->B[q * nb + b] * U[b * NS2 + s];
                Uq[q * NS2 + s] = acc;
            }
        /* VolumeFluxesFunctor, flux_functors_impl.h:46-115, dim 2 */
        for (int q = 0; q < nq; q++) {
            double U5[5], gF[15], gF1[8], gF2[8];
            embed(Uq + q * NS2, U5);
            orc_conv_flux(c->gamma, U5, gF);
            for (int d = 0; d < 2; d++) {
                gF1[d * NS2 + 0] = gF[d * 5 + 0];
                gF1[d * NS2 + 1] = gF[d * 5 + 1];
                gF1[d * NS2 + 2] = gF[d * 5 + 2];
                gF1[d * NS2 + 3] = gF[d * 5 + 4];
            }
            const double* ij = c->ijac + ((size_t)e * nq + q) * 4;
            const double dj = c->djac[(size_t)e * nq + q], w = c->vq_wts[q];
            for (int i = 0; i < 8; i++) gF2[i] = 0.;
            for (int d1 = 0; d1 < 2; d1++)
                for (int d2 = 0; d2 < 2; d2++)
                    for (int s = 0; s < NS2; s++) gF2[d1 * NS2 + s] += gF1[d2 * NS2 + s] * ij[d1 * 2 + d2] * dj * w;
            for (int d = 0; d < 2; d++)
                for (int s = 0; s < NS2; s++) vg[(q * NS2 + s) * 2 + d] = gF2[d * NS2 + s];
        }
        /* calculate_volume_flux_integral, solver/tools.cpp:7-35 */
        double* r = res + (size_t)e * nb * NS2;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS2; s++)
                for (int q = 0; q < nq; q++)
                    for (int d = 0; d < 2; d++) r[b * NS2 + s] += c->Dref[(q * nb + b) * 2 + d] * vg[(q * NS2 + s) * 2 + d];
        double* Uf = c->Uqf + (size_t)e * 4 * nqf * NS2;
        for (int q = 0; q < 4 * nqf; q++)
            for (int s = 0; s < NS2; s++) {
                double acc = 0.0;
                for (int b = 0; b < nb; b++) acc += c->Bf[q * nb + b] * U[b * NS2 + s];
                Uf[q * NS2 + s] = acc;
            }
    }
#pragma omp parallel for num_threads(nthreads()) schedule(static) reduction(+ : fails)
    for (int f = 0; f < nif; f++) {
        int eL = c->ifd[f * 6 + 0], fL = c->ifd[f * 6 + 1];
        int eR = c->ifd[f * 6 + 3], fR = c->ifd[f * 6 + 4];
        for (int q = 0; q < nqf; q++) {
            const double* UL = c->Uqf + (((size_t)eL * 4 + fL) * nqf + c->qidxL[f * nqf + q]) * NS2;
            const double* UR = c->Uqf + (((size_t)eR * 4 + fR) * nqf + c->qidxR[f * nqf + q]) * NS2;
            const double* N2 = c->normals + ((size_t)f * nqf + q) * 2;
            double uL[5], uR[5], N3[3] = {N2[0], N2[1], 0.0}, F5[5];
            embed(UL, uL);
            embed(UR, uR);
            if (orc_num_flux(c->flux_type, c->gamma, uL, uR, N3, F5)) fails++;
            double* Fq = c->Fq + ((size_t)f * nqf + q) * NS2;
            Fq[0] = F5[0] * c->fwts[q];
            Fq[1] = F5[1] * c->fwts[q];
            Fq[2] = F5[2] * c->fwts[q];
            Fq[3] = F5[4] * c->fwts[q];
        }
    }
    c->flux_fail += fails;
    for (int f = 0; f < nif; f++) {
        int eL = c->ifd[f * 6 + 0], fL = c->ifd[f * 6 + 1];
        int eR = c->ifd[f * 6 + 3], fR = c->ifd[f * 6 + 4];
        for (int q = 0; q < nqf; q++)
            for (int s = 0; s < NS2; s++) {
                double v = c->Fq[((size_t)f * nqf + q) * NS2 + s];
                c->Fq_elem[(((size_t)eL * 4 + fL) * nqf + c->qidxL[f * nqf + q]) * NS2 + s] = -1.0 * v;
                c->Fq_elem[(((size_t)eR * 4 + fR) * nqf + c->qidxR[f * nqf + q]) * NS2 + s] = v;
            }
    }
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int e = 0; e < ne; e++) {
        const double* Fe = c->Fq_elem + (size_t)e * 4 * nqf * NS2;
        double* r = res + (size_t)e * nb * NS2;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS2; s++) {
                double acc = 0.0;
                for (int q = 0; q < 4 * nqf; q++) acc += c->Bf[q * nb + b] * Fe[q * NS2 + s];
                r[b * NS2 + s] += acc;
            }
    }
}

static void mult_inv_mass(orc2_case* c, double dt, const double* res, double* dU)
{
    const int nb = c->nb;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int e = 0; e < c->ne; e++) {
        const double* iM = c->iMM + (size_t)e * nb * nb;
        const double* r = res + (size_t)e * nb * NS2;
        double* d = dU + (size_t)e * nb * NS2;
        for (int b = 0; b < nb; b++)
            for (int s = 0; s < NS2; s++) {
                double acc = 0.0;
                for (int k = 0; k < nb; k++) acc += iM[b * nb + k] * r[k * NS2 + s];
                d[b * NS2 + s] = dt * acc;
            }
    }
}

/* RK4<2>::take_time_step, stepper.cpp:71-142 */
void orc2_rk4_steps(orc2_case* c, double* Uc, double dt, int nsteps)
{
    const long n = (long)c->ne * c->nb * NS2;
    double *d1 = c->dU[0], *d2 = c->dU[1], *d3 = c->dU[2], *d4 = c->dU[3], *Uh = c->Uhold;
    for (int it = 0; it < nsteps; it++) {
        memcpy(Uh, Uc, sizeof(double) * n);
        orc2_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d1);
        for (long i = 0; i < n; i++) Uc[i] = 0.5 * d1[i] + 1.0 * Uh[i];
        orc2_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d2);
        for (long i = 0; i < n; i++) Uc[i] = 0.5 * d2[i] + 1.0 * Uh[i];
        orc2_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d3);
        for (long i = 0; i < n; i++) Uc[i] = 1.0 * d3[i] + 1.0 * Uh[i];
        orc2_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, d4);
        for (long i = 0; i < n; i++) {
            double a = d4[i] + 2.0 * d3[i];
            a = a + 2.0 * d2[i];
            a = a + 1.0 * d1[i];
            Uh[i] = Uh[i] + (1.0 / 6.0) * a;
            Uc[i] = Uh[i];
        }
    }
}

/* FE<2>::take_time_step, stepper.cpp:23-55 */
void orc2_fe_steps(orc2_case* c, double* Uc, double dt, int nsteps)
{
    const long n = (long)c->ne * c->nb * NS2;
    for (int it = 0; it < nsteps; it++) {
        orc2_residual(c, Uc, c->res);
        mult_inv_mass(c, dt, c->res, c->dU[0]);
        for (long i = 0; i < n; i++) Uc[i] = Uc[i] + 1.0 * c->dU[0][i];
    }
}

/* get_error, ord 2, volume-normalised, post/main.cpp:30-201 */
void orc2_l2_error(orc2_case* c, const double* Uc, double t, double* err)
{
    const int nb = c->nb, nq = c->nqe;
    double tot[NS2] = {0, 0, 0, 0};
    double* per = malloc(sizeof(double) * c->ne * NS2);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int e = 0; e < c->ne; e++) {
        double X[8], jac[4], Ue[NS2], Uq[NS2], xp[2];
        double acc[NS2] = {0, 0, 0, 0};
        elem_coords(c, e, X);
        const double* U = Uc + (size_t)e * nb * NS2;
        for (int q = 0; q < nq; q++) {
            for (int s = 0; s < NS2; s++) {
                double a = 0.0;
                for (int b = 0; b < nb; b++) a += c->Be[q * nb + b] * U[b * NS2 + s];
                Uq[s] = a;
            }
            for (int d = 0; d < 2; d++) {
                double s = 0.0;
                for (int n = 0; n < 4; n++) s += c->ge_val[q * 4 + n] * X[n * 2 + d];
                xp[d] = s;
            }
            ic2(c, xp, t, Ue);
            elem_jac(X, c->ge_grad + q * 8, jac);
            double dj = det2(jac);
            for (int s = 0; s < NS2; s++) {
                double d = Uq[s] - Ue[s];
                acc[s] += d * d * c->eq_wts[q] * dj;
            }
        }
        for (int s = 0; s < NS2; s++) per[e * NS2 + s] = acc[s];
    }
    for (int e = 0; e < c->ne; e++)
        for (int s = 0; s < NS2; s++) tot[s] += per[e * NS2 + s];
    free(per);
    double V = orc2_total_volume(c);
    for (int s = 0; s < NS2; s++) err[s] = sqrt(tot[s] / V);
}

void orc2_face_normals(const orc2_case* c, double* N)
{
    memcpy(N, c->normals, sizeof(double) * (size_t)c->nif * c->nqf * 2);
}
