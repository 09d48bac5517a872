// numerics.cpp -- see numerics.h.
#include "numerics.h"

#include <cmath>
#include <stdexcept>
#include <string>

namespace dgh {

int hex_quadrature_order(int order) { return 2 * (order + 1) + 1; }
int quad_quadrature_order(int order) { return (2 * order + 1) + 2; }
int points_per_direction(int qorder)
{
    // even orders round up to the same point count as the next odd order
    return (qorder % 2 == 0) ? (qorder + 2) / 2 : (qorder + 1) / 2;
}

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w)
{
    // Newton on the three-term recurrence of P_n, carried in long double and
    // rounded once; symmetric pairs are written from the positive root.
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < (n + 1) / 2; ++i) {
        long double z = std::cos(pi * (i + 0.75L) / (n + 0.5L));
        auto eval = [n](long double t, long double& pn, long double& dpn) {
            long double a = 1.0L, b = t;
            if (n == 0) { pn = 1.0L; dpn = 0.0L; return; }
            for (int k = 2; k <= n; ++k) {
                long double c = ((2.0L * k - 1.0L) * t * b - (k - 1.0L) * a) / k;
                a = b;
                b = c;
            }
            pn = b;
            dpn = n * (t * b - a) / (t * t - 1.0L);
        };
        long double pn, dpn;
        for (int it = 0; it < 200; ++it) {
            eval(z, pn, dpn);
            long double dz = pn / dpn;
            z -= dz;
            if (std::fabs(dz) < 1e-30L) break;
        }
        eval(z, pn, dpn);
        long double wi = 2.0L / ((1.0L - z * z) * dpn * dpn);
        if (2 * i + 1 == n) z = 0.0L;
        x[n - 1 - i] = static_cast<double>(z);
        x[i] = -static_cast<double>(z);
        w[i] = w[n - 1 - i] = static_cast<double>(wi);
    }
}

std::vector<double> equidistant_nodes(int nnodes)
{
    std::vector<double> xn(nnodes, 0.0);
    if (nnodes <= 1) return xn;
    const double dx = 2.0 / (static_cast<double>(nnodes) - 1.0);
    for (int i = 0; i < nnodes; ++i) xn[i] = -1.0 + static_cast<double>(i) * dx;
    return xn;
}

void lagrange_1d(double x, const std::vector<double>& xn, double* val, double* grad)
{
    const int nn = static_cast<int>(xn.size());
    if (nn == 1) {
        if (val) val[0] = 1.0;
        if (grad) grad[0] = 0.0;
        return;
    }
    for (int i = 0; i < nn; ++i) {
        if (val) {
            double v = 1.0;
            for (int j = 0; j < nn; ++j)
                if (j != i) v *= (x - xn[j]) / (xn[i] - xn[j]);
            val[i] = v;
        }
        if (grad) {
            double g = 0.0;
            for (int j = 0; j < nn; ++j) {
                if (j == i) continue;
                double prod = 1.0 / (xn[i] - xn[j]);
                for (int k = 0; k < nn; ++k)
                    if (k != i && k != j) prod *= (x - xn[k]) / (xn[i] - xn[k]);
                g += prod;
            }
            grad[i] = g;
        }
    }
}

// Corner nodes of each reference face with orientation 0, as listed by
// get_points_on_face_hexahedron (shape.cpp:236-272); corner c of the unit cube
// has coordinates (c&1, c&2, c&4) -> (+-1, +-1, +-1).
static const int kFaceCorners[6][4] = {
    {0, 2, 3, 1}, {0, 1, 5, 4}, {1, 3, 7, 5}, {3, 2, 6, 7}, {2, 0, 4, 6}, {4, 5, 7, 6}};

static double corner_coord(int c, int axis) { return ((c >> axis) & 1) ? 1.0 : -1.0; }

int face_axis(int f)
{
    for (int a = 0; a < 3; ++a) {
        double v = corner_coord(kFaceCorners[f][0], a);
        bool same = true;
        for (int k = 1; k < 4; ++k) same = same && corner_coord(kFaceCorners[f][k], a) == v;
        if (same) return a;
    }
    throw std::logic_error("degenerate face table");
}

int face_side(int f) { return corner_coord(kFaceCorners[f][0], face_axis(f)) > 0 ? 1 : 0; }

void face_canonical_map(int m, int f, std::vector<int>& canon)
{
    std::vector<double> s, w;
    gauss_legendre(m, s, w);
    const int ax = face_axis(f);
    const int a0 = ax == 0 ? 1 : 0;
    const int a1 = ax == 2 ? 1 : 2;
    canon.assign(m * m, -1);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) {
            // bilinear corner map (barycentric weights of shape.cpp:304-323)
            long double xb = (s[i] + 1.0L) / 2.0L, yb = (s[j] + 1.0L) / 2.0L;
            long double b[4] = {(1 - xb) * (1 - yb), xb * (1 - yb), xb * yb, (1 - xb) * yb};
            long double P[3] = {0, 0, 0};
            for (int k = 0; k < 4; ++k)
                for (int a = 0; a < 3; ++a) P[a] += b[k] * corner_coord(kFaceCorners[f][k], a);
            int t0 = -1, t1 = -1;
            for (int t = 0; t < m; ++t) {
                if (std::fabs(static_cast<double>(P[a0]) - s[t]) < 1e-12) t0 = t;
                if (std::fabs(static_cast<double>(P[a1]) - s[t]) < 1e-12) t1 = t;
            }
            if (t0 < 0 || t1 < 0) throw std::logic_error("face point off the GL grid");
            canon[j * m + i] = t1 * m + t0;
        }
}

void face_orientation_order(int orient, int npts, std::vector<int>& order)
{
    // The eight dihedral re-orderings of an n1 x n1 face grid, written as
    // closed-form index maps of (row, col) = (q / n1, q % n1); they reproduce
    // the walk-based listing of shape.cpp:336-423.
    const int n1 = static_cast<int>(std::lround(std::sqrt(static_cast<double>(npts))));
    order.assign(npts, 0);
    for (int q = 0; q < npts; ++q) {
        const int r = q / n1, c = q % n1, R = n1 - 1 - r, C = n1 - 1 - c;
        int v = 0;
        switch (orient) {
            case 0: v = r * n1 + c; break;          // identity
            case 1: v = c * n1 + R; break;          // quarter turn
            case 2: v = R * n1 + C; break;          // half turn
            case 3: v = C * n1 + r; break;          // three-quarter turn
            case 4: v = c * n1 + r; break;          // transpose
            case 5: v = r * n1 + C; break;          // mirror of columns
            case 6: v = C * n1 + R; break;          // anti-transpose
            case 7: v = R * n1 + c; break;          // mirror of rows
            default: throw std::invalid_argument("orientation must be 0..7");
        }
        order[q] = v;
    }
}

std::array<int, 4> face_geometry_nodes(int f)
{
    // i0 + i*d0 + j*d1 for gorder = 1 (shape.cpp:436-479)
    static const int t[6][3] = {{0, 2, 1}, {0, 1, 4}, {1, 2, 4}, {3, -1, 4}, {2, -2, 4}, {4, 1, 2}};
    std::array<int, 4> nodes{};
    for (int j = 0, k = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i, ++k) nodes[k] = t[f][0] + i * t[f][1] + j * t[f][2];
    return nodes;
}

static void invert_ld(int n, std::vector<long double> a, std::vector<double>& inv)
{
    std::vector<long double> b(n * n, 0.0L);
    for (int i = 0; i < n; ++i) b[i * n + i] = 1.0L;
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[i * n + k]) > std::fabs(a[piv * n + k])) piv = i;
        for (int j = 0; j < n; ++j) {
            std::swap(a[k * n + j], a[piv * n + j]);
            std::swap(b[k * n + j], b[piv * n + j]);
        }
        long double d = a[k * n + k];
        for (int j = 0; j < n; ++j) { a[k * n + j] /= d; b[k * n + j] /= d; }
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            long double f = a[i * n + k];
            for (int j = 0; j < n; ++j) { a[i * n + j] -= f * a[k * n + j]; b[i * n + j] -= f * b[k * n + j]; }
        }
    }
    inv.resize(n * n);
    for (int i = 0; i < n * n; ++i) inv[i] = static_cast<double>(b[i]);
}

Tables1D make_tables(int p)
{
    if (p < 0 || p > 8) throw std::invalid_argument("order out of range: " + std::to_string(p));
    Tables1D t;
    t.p = p;
    t.n = p + 1;
    t.m = points_per_direction(hex_quadrature_order(p));  // = p + 2
    const auto xn = equidistant_nodes(t.n);
    gauss_legendre(t.m, t.xq, t.wq);
    t.B.assign(t.m * t.n, 0.0);
    t.D.assign(t.m * t.n, 0.0);
    for (int q = 0; q < t.m; ++q) lagrange_1d(t.xq[q], xn, &t.B[q * t.n], &t.D[q * t.n]);

    // 1D mass matrix on the inverse-mass rule (order 2p, helpers.cpp:57-58):
    // the 3D reference mass matrix is its Kronecker cube for affine elements.
    const int mm = points_per_direction(hex_quadrature_order(2 * p));
    std::vector<double> xm, wm;
    gauss_legendre(mm, xm, wm);
    std::vector<long double> M(t.n * t.n, 0.0L);
    std::vector<double> phi(t.n);
    for (int q = 0; q < mm; ++q) {
        lagrange_1d(xm[q], xn, phi.data(), nullptr);
        for (int i = 0; i < t.n; ++i)
            for (int j = 0; j < t.n; ++j) M[i * t.n + j] += (long double)wm[q] * phi[i] * phi[j];
    }
    invert_ld(t.n, M, t.Minv);

    // IC / error rule: order 2*max(p,1) (base.cpp:128-131, post/main.cpp:64-67)
    t.me = points_per_direction(hex_quadrature_order(2 * (p > 1 ? p : 1)));
    gauss_legendre(t.me, t.xe, t.we);
    t.Be.assign(t.me * t.n, 0.0);
    for (int q = 0; q < t.me; ++q) lagrange_1d(t.xe[q], xn, &t.Be[q * t.n], nullptr);
    // the inverse-mass rule's 1D tables, for general (trilinear) elements
    t.mm = mm;
    t.xm = xm;
    t.wm = wm;
    t.Bm.assign(t.mm * t.n, 0.0);
    for (int q = 0; q < t.mm; ++q) lagrange_1d(t.xm[q], xn, &t.Bm[q * t.n], nullptr);
    return t;
}

void trilinear_jacobian(const double* X, const double* xi, double* jac)
{
    // geometric basis phi_n = prod_a (1 + s_a(n) xi_a) / 2, node n = i + 2j + 4k
    double dphi[8][3];
    for (int n = 0; n < 8; ++n)
        for (int j = 0; j < 3; ++j) {
            double g = 1.0;
            for (int a = 0; a < 3; ++a) {
                const double s = ((n >> a) & 1) ? 1.0 : -1.0;
                g *= a == j ? 0.5 * s : 0.5 * (1.0 + s * xi[a]);
            }
            dphi[n][j] = g;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int n = 0; n < 8; ++n) s += X[n * 3 + i] * dphi[n][j];
            jac[i * 3 + j] = s;
        }
}

double det3(const double* M)
{
    return M[0] * M[4] * M[8] - M[0] * M[5] * M[7] - M[1] * M[3] * M[8] + M[1] * M[5] * M[6] + M[2] * M[3] * M[7] -
           M[2] * M[4] * M[6];
}

bool general_inverse_mass(const Tables1D& t, const double* X, double* out)
{
    const int n = t.n, mm = t.mm, nb = n * n * n;
    // w * det J at the mass points, [z][y][x]
    std::vector<double> D(static_cast<size_t>(mm) * mm * mm);
    for (int z = 0; z < mm; ++z)
        for (int y = 0; y < mm; ++y)
            for (int x = 0; x < mm; ++x) {
                const double xi[3] = {t.xm[x], t.xm[y], t.xm[z]};
                double jac[9];
                trilinear_jacobian(X, xi, jac);
                D[(static_cast<size_t>(z) * mm + y) * mm + x] = t.wm[x] * t.wm[y] * t.wm[z] * det3(jac);
            }
    // sum-factorised B^T D B: contract x, then y, then z (basis index c*n*n + b*n + a)
    std::vector<double> T1(static_cast<size_t>(n) * n * mm * mm);  // [a][a'][z][y]
    for (int a = 0; a < n; ++a)
        for (int a2 = 0; a2 < n; ++a2)
            for (int z = 0; z < mm; ++z)
                for (int y = 0; y < mm; ++y) {
                    double s = 0.0;
                    for (int x = 0; x < mm; ++x)
                        s += t.Bm[x * n + a] * t.Bm[x * n + a2] * D[(static_cast<size_t>(z) * mm + y) * mm + x];
                    T1[((static_cast<size_t>(a) * n + a2) * mm + z) * mm + y] = s;
                }
    std::vector<double> T2(static_cast<size_t>(n) * n * n * n * mm);  // [a][a'][b][b'][z]
    for (int aa = 0; aa < n * n; ++aa)
        for (int b = 0; b < n; ++b)
            for (int b2 = 0; b2 < n; ++b2)
                for (int z = 0; z < mm; ++z) {
                    double s = 0.0;
                    for (int y = 0; y < mm; ++y)
                        s += t.Bm[y * n + b] * t.Bm[y * n + b2] * T1[(static_cast<size_t>(aa) * mm + z) * mm + y];
                    T2[((static_cast<size_t>(aa) * n + b) * n + b2) * mm + z] = s;
                }
    std::vector<double> M(static_cast<size_t>(nb) * nb);
    for (int a = 0; a < n; ++a)
        for (int a2 = 0; a2 < n; ++a2)
            for (int b = 0; b < n; ++b)
                for (int b2 = 0; b2 < n; ++b2)
                    for (int c = 0; c < n; ++c)
                        for (int c2 = 0; c2 < n; ++c2) {
                            double s = 0.0;
                            const double* t2 = &T2[(((static_cast<size_t>(a) * n + a2) * n + b) * n + b2) * mm];
                            for (int z = 0; z < mm; ++z) s += t.Bm[z * n + c] * t.Bm[z * n + c2] * t2[z];
                            M[static_cast<size_t>((c * n + b) * n + a) * nb + (c2 * n + b2) * n + a2] = s;
                        }
    // unpivoted LU (Doolittle, unit lower L), then the inverse column by column
    for (int k = 0; k < nb; ++k) {
        const double piv = M[static_cast<size_t>(k) * nb + k];
        if (!(std::fabs(piv) > 0.0)) return false;
        for (int i = k + 1; i < nb; ++i) M[static_cast<size_t>(i) * nb + k] /= piv;
        for (int i = k + 1; i < nb; ++i) {
            const double lik = M[static_cast<size_t>(i) * nb + k];
            for (int j = k + 1; j < nb; ++j) M[static_cast<size_t>(i) * nb + j] -= lik * M[static_cast<size_t>(k) * nb + j];
        }
    }
    std::vector<double> col(nb);
    for (int c = 0; c < nb; ++c) {
        for (int i = 0; i < nb; ++i) {
            double s = i == c ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= M[static_cast<size_t>(i) * nb + k] * col[k];
            col[i] = s;
        }
        for (int i = nb - 1; i >= 0; --i) {
            double s = col[i];
            for (int k = i + 1; k < nb; ++k) s -= M[static_cast<size_t>(i) * nb + k] * col[k];
            col[i] = s / M[static_cast<size_t>(i) * nb + i];
        }
        // column c of the inverse: iMM[i][c] = col[i], stored at out[c * nb + i]
        for (int i = 0; i < nb; ++i) out[static_cast<size_t>(c) * nb + i] = col[i];
    }
    return true;
}

}  // namespace dgh
