// mesh.cpp -- see mesh.h.
#include "mesh.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <stdexcept>

#include "numerics.h"

namespace dgh {

namespace {

// reference corner l of the unit cube: (+-1, +-1, +-1), x fastest
inline int corner_sign(int l, int a) { return ((l >> a) & 1) ? 1 : -1; }

// The 24 proper rotations of the cube as signed permutation matrices.
std::vector<std::array<int, 9>> cube_rotations()
{
    std::vector<std::array<int, 9>> rots;
    const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (const auto& pm : perms)
        for (int sg = 0; sg < 8; ++sg) {
            std::array<int, 9> R{};
            for (int r = 0; r < 3; ++r) R[r * 3 + pm[r]] = (sg >> r) & 1 ? -1 : 1;
            const int det = R[0] * (R[4] * R[8] - R[5] * R[7]) - R[1] * (R[3] * R[8] - R[5] * R[6]) +
                            R[2] * (R[3] * R[7] - R[4] * R[6]);
            if (det == 1) rots.push_back(R);
        }
    return rots;
}

// physical position of reference point xi in an element (trilinear map)
void ref_to_phys(const double* X /*[8][3]*/, const double* xi, double* x)
{
    x[0] = x[1] = x[2] = 0.0;
    for (int l = 0; l < 8; ++l) {
        double w = 1.0;
        for (int a = 0; a < 3; ++a) w *= 0.5 * (1.0 + corner_sign(l, a) * xi[a]);
        for (int a = 0; a < 3; ++a) x[a] += w * X[l * 3 + a];
    }
}

// face points (orientation 0) of reference face f on an m x m GL grid, in the
// reference's face-point order, as reference-cube coordinates
void face_ref_points(int m, int f, std::vector<double>& xi)
{
    std::vector<double> s, w;
    gauss_legendre(m, s, w);
    std::vector<int> canon;
    face_canonical_map(m, f, canon);
    const int ax = face_axis(f);
    const int a0 = ax == 0 ? 1 : 0, a1 = ax == 2 ? 1 : 2;
    xi.assign(m * m * 3, 0.0);
    for (int q = 0; q < m * m; ++q) {
        xi[q * 3 + ax] = face_side(f) ? 1.0 : -1.0;
        xi[q * 3 + a0] = s[canon[q] % m];
        xi[q * 3 + a1] = s[canon[q] / m];
    }
}

}  // namespace

BoxMesh make_periodic_box(const int n[3], const double x0[3], const double len[3], unsigned rotate_seed)
{
    BoxMesh b;
    const int nx = n[0], ny = n[1], nz = n[2];
    if (nx < 1 || ny < 1 || nz < 1) throw std::invalid_argument("box needs >= 1 element per direction");
    b.nnode = (nx + 1) * (ny + 1) * (nz + 1);
    b.nelem = nx * ny * nz;
    b.nface = 3 * b.nelem;
    b.coords.resize(static_cast<size_t>(b.nnode) * 3);
    auto node_id = [&](int i, int j, int k) { return static_cast<unsigned>(i + (nx + 1) * (j + (ny + 1) * k)); };
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                const size_t id = node_id(i, j, k);
                b.coords[id * 3 + 0] = x0[0] + len[0] * i / nx;
                b.coords[id * 3 + 1] = x0[1] + len[1] * j / ny;
                b.coords[id * 3 + 2] = x0[2] + len[2] * k / nz;
            }
    const auto rots = cube_rotations();
    std::vector<int> rot_of(b.nelem, -1);  // -1: identity numbering
    uint64_t st = rotate_seed;
    for (int e = 0; e < b.nelem; ++e) {
        if (rotate_seed) {
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            rot_of[e] = static_cast<int>((st >> 33) % rots.size());
        }
    }
    b.e2n.resize(static_cast<size_t>(b.nelem) * 8);
    auto elem_id = [&](int i, int j, int k) { return i + nx * (j + ny * k); };
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const int e = elem_id(i, j, k);
                for (int l = 0; l < 8; ++l) {
                    int o[3];
                    for (int a = 0; a < 3; ++a) {
                        int v = corner_sign(l, a);
                        if (rot_of[e] >= 0) {
                            const auto& R = rots[rot_of[e]];
                            v = R[a * 3 + 0] * corner_sign(l, 0) + R[a * 3 + 1] * corner_sign(l, 1) +
                                R[a * 3 + 2] * corner_sign(l, 2);
                        }
                        o[a] = (v + 1) / 2;
                    }
                    b.e2n[static_cast<size_t>(e) * 8 + l] = node_id(i + o[0], j + o[1], k + o[2]);
                }
            }

    // local face of element e whose outward normal is +-axis `a` physically
    auto local_face = [&](int e, int a, int sign) {
        for (int f = 0; f < 6; ++f) {
            int nref[3] = {0, 0, 0};
            nref[face_axis(f)] = face_side(f) ? 1 : -1;
            int nphys[3] = {nref[0], nref[1], nref[2]};
            if (rot_of[e] >= 0) {
                const auto& R = rots[rot_of[e]];
                for (int r = 0; r < 3; ++r) nphys[r] = R[r * 3 + 0] * nref[0] + R[r * 3 + 1] * nref[1] + R[r * 3 + 2] * nref[2];
            }
            if (nphys[a] == sign) return f;
        }
        throw std::logic_error("no face with that normal");
    };
    auto elem_X = [&](int e, double* X) {
        for (int l = 0; l < 8; ++l)
            for (int a = 0; a < 3; ++a) X[l * 3 + a] = b.coords[static_cast<size_t>(b.e2n[static_cast<size_t>(e) * 8 + l]) * 3 + a];
    };
    // orientations are matched on a 3 x 3 face grid: every dihedral map of it is distinct
    const int mo = 3;
    std::vector<double> fxi[6];
    for (int f = 0; f < 6; ++f) face_ref_points(mo, f, fxi[f]);
    std::vector<int> orders[8];
    for (int o = 0; o < 8; ++o) face_orientation_order(o, mo * mo, orders[o]);

    b.faces.resize(static_cast<size_t>(b.nface) * 8);
    int fi = 0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                for (int a = 0; a < 3; ++a) {
                    const int eL = elem_id(i, j, k);
                    int ii = i, jj = j, kk = k;
                    if (a == 0) ii = (i + 1) % nx;
                    if (a == 1) jj = (j + 1) % ny;
                    if (a == 2) kk = (k + 1) % nz;
                    const int eR = elem_id(ii, jj, kk);
                    const int fL = local_face(eL, a, +1), fR = local_face(eR, a, -1);
                    double XL[24], XR[24];
                    elem_X(eL, XL);
                    elem_X(eR, XR);
                    std::vector<double> PL(mo * mo * 3), PR(mo * mo * 3);
                    for (int q = 0; q < mo * mo; ++q) {
                        ref_to_phys(XL, &fxi[fL][q * 3], &PL[q * 3]);
                        ref_to_phys(XR, &fxi[fR][q * 3], &PR[q * 3]);
                    }
                    int oR = -1;
                    for (int o = 0; o < 8 && oR < 0; ++o) {
                        bool ok = true;
                        for (int q = 0; q < mo * mo && ok; ++q)
                            for (int c = 0; c < 3 && ok; ++c) {
                                double d = PL[q * 3 + c] - PR[orders[o][q] * 3 + c];
                                d -= len[c] * std::round(d / len[c]);
                                ok = std::fabs(d) < 1e-9 * len[c];
                            }
                        if (ok) oR = o;
                    }
                    if (oR < 0) throw std::logic_error("face points of neighbours do not match");
                    unsigned* row = &b.faces[static_cast<size_t>(fi) * 8];
                    row[0] = 0; row[1] = eL; row[2] = fL; row[3] = 0;
                    row[4] = 0; row[5] = eR; row[6] = fR; row[7] = static_cast<unsigned>(oR);
                    ++fi;
                }
    return b;
}

// General geometry, volume part: node coordinates, ijac * djac at the volume
// GL points (BasisTools::get_element_jacobian, basis/tools.cpp:42-66, with the
// closed-form Math::det / Math::invA, linear_algebra.cpp:108-122, 243-259),
// element volumes on that rule (MeshTools::get_element_volume,
// mesh/tools.cpp:28-36) and shortest edges; one placeholder affine class.
static std::string prepare_general_volume(const MeshView& mv, int m, PreparedMesh& out)
{
    const int ne = mv.nelem, nq = m * m * m;
    std::vector<double> x, w;
    gauss_legendre(m, x, w);
    out.gnodes.resize(static_cast<size_t>(ne) * 24);
    out.gjd.resize(static_cast<size_t>(ne) * 9 * nq);
    out.elem_h.resize(ne);
    std::vector<double> vol(ne, 0.0);
    int bad = -1;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; ++e) {
        double* X = &out.gnodes[static_cast<size_t>(e) * 24];
        for (int l = 0; l < 8; ++l)
            for (int a = 0; a < 3; ++a)
                X[l * 3 + a] = mv.coords[static_cast<size_t>(mv.e2n[static_cast<size_t>(e) * 8 + l]) * 3 + a];
        double v = 0.0;
        for (int q = 0; q < nq; ++q) {
            const int qx = q % m, qy = (q / m) % m, qz = q / (m * m);
            const double xi[3] = {x[qx], x[qy], x[qz]};
            double M[9];
            trilinear_jacobian(X, xi, M);
            const double det = det3(M);
            if (!(det > 0.0)) {
#pragma omp critical
                bad = bad < 0 ? e : std::min(bad, e);
                break;
            }
            double inv[9];
            inv[0] = (M[4] * M[8] - M[5] * M[7]) / det;
            inv[3] = -(M[3] * M[8] - M[5] * M[6]) / det;
            inv[6] = (M[3] * M[7] - M[4] * M[6]) / det;
            inv[1] = -(M[1] * M[8] - M[2] * M[7]) / det;
            inv[4] = (M[0] * M[8] - M[2] * M[6]) / det;
            inv[7] = -(M[0] * M[7] - M[1] * M[6]) / det;
            inv[2] = (M[1] * M[5] - M[2] * M[4]) / det;
            inv[5] = -(M[0] * M[5] - M[2] * M[3]) / det;
            inv[8] = (M[0] * M[4] - M[1] * M[3]) / det;
            for (int k = 0; k < 9; ++k) out.gjd[(static_cast<size_t>(e) * 9 + k) * nq + q] = inv[k] * det;
            v += w[qx] * w[qy] * w[qz] * det;
        }
        vol[e] = v;
        double h = 1e300;
        for (int l = 0; l < 8; ++l)
            for (int a = 0; a < 3; ++a)
                if (!((l >> a) & 1)) {
                    const int l2 = l | (1 << a);
                    double d2 = 0.0;
                    for (int c = 0; c < 3; ++c) d2 += (X[l2 * 3 + c] - X[l * 3 + c]) * (X[l2 * 3 + c] - X[l * 3 + c]);
                    h = std::fmin(h, std::sqrt(d2));
                }
        out.elem_h[e] = h;
    }
    if (bad >= 0) return "element " + std::to_string(bad) + " has a non-positive Jacobian";
    out.volume = 0.0;
    out.hmin = 1e300;
    for (int e = 0; e < out.nowned; ++e) {
        out.volume += vol[e];
        out.hmin = std::fmin(out.hmin, out.elem_h[e]);
    }
    GeoClass g{};
    for (int i = 0; i < 3; ++i) g.J[i * 4] = g.JD[i * 4] = 1.0;
    g.djac = g.inv_djac = 1.0;
    for (int f = 0; f < 6; ++f) {
        g.nmag[f] = 1.0;
        g.N[f][face_axis(f)] = g.nhat[f][face_axis(f)] = g.nunit[f][face_axis(f)] = 1.0;
    }
    out.classes.assign(1, g);
    out.geo_class.assign(ne, 0);
    return "";
}

// General geometry, face part: the reference's face normals (precompute_normals,
// helpers.cpp:380-500 with shape.cpp:482-532): at face-loop point q the cross
// product of the tangents of the left element's bilinear face map (nodes in
// get_local_nodes_on_face_hexahedron order) at the first two coordinates of
// reference face 0's q-th point; each owned side stores it at its own
// canonical point of loop index q.
static void general_face_normals(const MeshView& mv, int m, const std::vector<int>* canon_inv,
                                 const std::vector<int>* order_inv, PreparedMesh& out)
{
    const int nf = m * m, nowned = out.nowned;
    std::vector<double> x, w;
    gauss_legendre(m, x, w);
    out.gN.assign(static_cast<size_t>(nowned) * 6 * 3 * nf, 0.0);
    std::vector<double> Nq(static_cast<size_t>(nf) * 3);
    for (int i = 0; i < mv.nface; ++i) {
        const unsigned* r = &mv.faces[static_cast<size_t>(i) * 8];
        const int eL = r[1], fL = r[2], oL = r[3], eR = r[5], fR = r[6], oR = r[7];
        if (eL >= nowned && eR >= nowned) continue;
        const auto nd = face_geometry_nodes(fL);
        const double* X = &out.gnodes[static_cast<size_t>(eL) * 24];
        for (int q = 0; q < nf; ++q) {
            // face 0's point q = j*m + i is (x[j], x[i], -1) in the reference cube
            const double s = x[q / m], t = x[q % m];
            double a[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < 4; ++k) {
                const int ii = k & 1, jj = k >> 1;
                const double vs = ii ? 0.5 * (1.0 + s) : 0.5 * (1.0 - s), gs = ii ? 0.5 : -0.5;
                const double vt = jj ? 0.5 * (1.0 + t) : 0.5 * (1.0 - t), gt = jj ? 0.5 : -0.5;
                for (int d = 0; d < 3; ++d) {
                    a[d] += X[nd[k] * 3 + d] * (gs * vt);
                    b[d] += X[nd[k] * 3 + d] * (vs * gt);
                }
            }
            Nq[q * 3 + 0] = a[1] * b[2] - a[2] * b[1];
            Nq[q * 3 + 1] = a[2] * b[0] - a[0] * b[2];
            Nq[q * 3 + 2] = a[0] * b[1] - a[1] * b[0];
        }
        const int side_e[2] = {eL, eR}, side_f[2] = {fL, fR}, side_o[2] = {oL, oR};
        for (int sd = 0; sd < 2; ++sd) {
            const int e = side_e[sd], f = side_f[sd], o = side_o[sd];
            if (e >= nowned) continue;
            for (int c = 0; c < nf; ++c) {
                const int q = order_inv[o][canon_inv[f][c]];
                for (int d = 0; d < 3; ++d)
                    out.gN[((static_cast<size_t>(e) * 6 + f) * 3 + d) * nf + c] = Nq[static_cast<size_t>(q) * 3 + d];
            }
        }
    }
}

std::string prepare_mesh(const MeshView& mv, int m, PreparedMesh& out)
{
    if (mv.nelem <= 0) return "mesh has no elements";
    if (mv.nnode <= 0 || !mv.coords || !mv.e2n) return "mesh arrays missing";
    if (mv.nface <= 0 || !mv.faces) return "unsupported: mesh has no interior faces";
    if (m < 2 || m > 16) return "face grid size out of range";
    const int ne = mv.nelem;
    out = PreparedMesh{};
    out.ne = ne;
    out.m = m;
    out.nowned = mv.nowned < 0 ? ne : mv.nowned;

    // ---- geometry: affine check and classes ----
    std::vector<double> Jall(static_cast<size_t>(ne) * 9);
    out.X0.resize(static_cast<size_t>(ne) * 3);
    double hs = 0.0;
    bool nonaffine = false;
    for (int e = 0; e < ne; ++e) {
        double X[24];
        for (int l = 0; l < 8; ++l) {
            const unsigned nid = mv.e2n[static_cast<size_t>(e) * 8 + l];
            if (nid >= static_cast<unsigned>(mv.nnode)) return "element node id out of range";
            for (int a = 0; a < 3; ++a) {
                X[l * 3 + a] = mv.coords[static_cast<size_t>(nid) * 3 + a];
                if (!std::isfinite(X[l * 3 + a])) return "element " + std::to_string(e) + " has a non-finite node coordinate";
            }
        }
        double* J = &Jall[static_cast<size_t>(e) * 9];
        for (int i = 0; i < 3; ++i) {
            J[i * 3 + 0] = 0.5 * (X[1 * 3 + i] - X[0 * 3 + i]);
            J[i * 3 + 1] = 0.5 * (X[2 * 3 + i] - X[0 * 3 + i]);
            J[i * 3 + 2] = 0.5 * (X[4 * 3 + i] - X[0 * 3 + i]);
        }
        double scale = 0.0;
        for (int i = 0; i < 9; ++i) scale = std::fmax(scale, std::fabs(J[i]));
        hs = std::fmax(hs, scale);
        for (int l = 0; l < 8; ++l)
            for (int i = 0; i < 3; ++i) {
                double v = X[i];
                for (int a = 0; a < 3; ++a) v += J[i * 3 + a] * (corner_sign(l, a) + 1);
                if (std::fabs(v - X[l * 3 + i]) > 1e-9 * scale) nonaffine = true;
            }
        for (int a = 0; a < 3; ++a) out.X0[static_cast<size_t>(e) * 3 + a] = X[a];
    }
    out.general = nonaffine;
    std::string gerr = out.general ? prepare_general_volume(mv, m, out) : std::string();
    if (!gerr.empty()) return gerr;
    if (!out.general) {
        std::map<std::array<long long, 10>, int> class_of;
        out.geo_class.resize(ne);
        out.hmin = 1e300;
        for (int e = 0; e < ne; ++e) {
            const double* J = &Jall[static_cast<size_t>(e) * 9];
            std::array<long long, 10> key{};
            for (int i = 0; i < 9; ++i) key[i] = std::llround(J[i] / hs * 68719476736.0);  // 2^36
            key[9] = mv.tag ? mv.tag[e] : 0;
            auto it = class_of.find(key);
            if (it != class_of.end()) {
                out.geo_class[e] = it->second;
                continue;
            }
            GeoClass g{};
            for (int i = 0; i < 9; ++i) g.J[i] = J[i];
            // Math::det / Math::invA closed forms (src/math/linear_algebra.cpp:108-122, 243-259)
            const double* M = J;
            const double det = M[0] * M[4] * M[8] - M[0] * M[5] * M[7] - M[1] * M[3] * M[8] +
                               M[1] * M[5] * M[6] + M[2] * M[3] * M[7] - M[2] * M[4] * M[6];
            if (!(det > 0.0)) return "element " + std::to_string(e) + " has a non-positive Jacobian";
            double inv[9];
            inv[0] = (M[4] * M[8] - M[5] * M[7]) / det;
            inv[3] = -(M[3] * M[8] - M[5] * M[6]) / det;
            inv[6] = (M[3] * M[7] - M[4] * M[6]) / det;
            inv[1] = -(M[1] * M[8] - M[2] * M[7]) / det;
            inv[4] = (M[0] * M[8] - M[2] * M[6]) / det;
            inv[7] = -(M[0] * M[7] - M[1] * M[6]) / det;
            inv[2] = (M[1] * M[5] - M[2] * M[4]) / det;
            inv[5] = -(M[0] * M[5] - M[2] * M[3]) / det;
            inv[8] = (M[0] * M[4] - M[1] * M[3]) / det;
            for (int i = 0; i < 9; ++i) g.JD[i] = inv[i] * det;
            g.djac = det;
            g.inv_djac = 1.0 / det;
            // face normals: cross product of the face map's tangent vectors built
            // from the face's geometry nodes (shape.cpp:482-532; sign +1 = outward
            // from the owning element, helpers.cpp:440-446)
            for (int f = 0; f < 6; ++f) {
                const auto nd = face_geometry_nodes(f);
                double t1[3], t2[3];
                for (int i = 0; i < 3; ++i) {
                    t1[i] = 0.0;
                    t2[i] = 0.0;
                    for (int a = 0; a < 3; ++a) {
                        t1[i] += J[i * 3 + a] * 0.5 * (corner_sign(nd[1], a) - corner_sign(nd[0], a));
                        t2[i] += J[i * 3 + a] * 0.5 * (corner_sign(nd[2], a) - corner_sign(nd[0], a));
                    }
                }
                g.N[f][0] = t1[1] * t2[2] - t1[2] * t2[1];
                g.N[f][1] = t1[2] * t2[0] - t1[0] * t2[2];
                g.N[f][2] = t1[0] * t2[1] - t1[1] * t2[0];
                double nm = 0.0;
                for (int d = 0; d < 3; ++d) nm += g.N[f][d] * g.N[f][d];
                nm = std::sqrt(nm);
                const double inv = 1. / nm;
                g.nmag[f] = nm;
                for (int d = 0; d < 3; ++d) {
                    g.nhat[f][d] = g.N[f][d] / nm;
                    g.nunit[f][d] = g.N[f][d] * inv;
                }
            }
            const int cid = static_cast<int>(out.classes.size());
            out.classes.push_back(g);
            class_of[key] = cid;
            out.geo_class[e] = cid;
        }
        out.volume = 0.0;
        for (int e = 0; e < (mv.nowned < 0 ? ne : std::min(mv.nowned, ne)); ++e) {  // owned elements
            const GeoClass& g = out.classes[out.geo_class[e]];
            out.volume += 8.0 * g.djac;
            for (int a = 0; a < 3; ++a) {
                const double len = 2.0 * std::sqrt(g.J[0 * 3 + a] * g.J[0 * 3 + a] + g.J[1 * 3 + a] * g.J[1 * 3 + a] +
                                                   g.J[2 * 3 + a] * g.J[2 * 3 + a]);
                out.hmin = std::fmin(out.hmin, len);
            }
        }

    }

    // ---- face gather table ----
    std::vector<int> canon[6], canon_inv[6];
    for (int f = 0; f < 6; ++f) {
        face_canonical_map(m, f, canon[f]);
        canon_inv[f].assign(m * m, -1);
        for (int q = 0; q < m * m; ++q) canon_inv[f][canon[f][q]] = q;
    }
    std::vector<int> order[8], order_inv[8];
    for (int o = 0; o < 8; ++o) {
        face_orientation_order(o, m * m, order[o]);
        order_inv[o].assign(m * m, -1);
        for (int q = 0; q < m * m; ++q) order_inv[o][order[o][q]] = q;
    }
    out.conn.assign(static_cast<size_t>(ne) * 12, -1);
    std::map<std::array<int, 4>, int> code_of;
    auto add_side = [&](int e, int f, int en, int fn, int ox, int oy, int isL) -> std::string {
        int* slot = &out.conn[(static_cast<size_t>(e) * 6 + f) * 2];
        if (slot[0] != -1) return "face " + std::to_string(f) + " of element " + std::to_string(e) + " listed twice";
        std::array<int, 4> key{f, fn, ox, oy};
        auto it = code_of.find(key);
        int code;
        if (it == code_of.end()) {
            code = static_cast<int>(code_of.size());
            code_of[key] = code;
            for (int c = 0; c < m * m; ++c) {
                const int a = canon_inv[f][c];        // own face point (reference order)
                const int q = order_inv[ox][a];       // face-loop index (quad_idx, helpers.cpp:358-368)
                const int b = order[oy][q];           // neighbour's face point
                out.cmap.push_back(static_cast<uint8_t>(canon[fn][b]));
            }
        } else {
            code = it->second;
        }
        if (code >= (1 << 27)) return "too many face codes";
        slot[0] = en;
        slot[1] = fn | (isL << 3) | (code << 4);
        return "";
    };
    const int nowned = mv.nowned < 0 ? ne : mv.nowned;
    if (nowned > ne || nowned < 1) return "owned element count out of range";
    for (int e = 0; mv.elem_rank && e < nowned; ++e)
        if (mv.elem_rank[e] != mv.rank) return "owned element " + std::to_string(e) + " has another rank";
    for (int i = 0; i < mv.nface; ++i) {
        const unsigned* r = &mv.faces[static_cast<size_t>(i) * 8];
        // the entries are unsigned: compared as such, a negative value written
        // into the table is a huge one, not a small one
        if (r[1] >= static_cast<unsigned>(ne) || r[5] >= static_cast<unsigned>(ne) || r[2] > 5u || r[6] > 5u ||
            r[3] > 7u || r[7] > 7u)
            return "face " + std::to_string(i) + " has an out-of-range entry";
        const int eL = r[1], fL = r[2], oL = r[3], eR = r[5], fR = r[6], oR = r[7];
        if (!mv.elem_rank) {
            if (static_cast<int>(r[0]) != mv.rank || static_cast<int>(r[4]) != mv.rank)
                return "unsupported: face " + std::to_string(i) + " crosses ranks (single-GPU build)";
        } else if (static_cast<int>(r[0]) != mv.elem_rank[eL] || static_cast<int>(r[4]) != mv.elem_rank[eR]) {
            return "face " + std::to_string(i) + " names a rank that does not own its element";
        }
        if (eL >= nowned && eR >= nowned) return "face " + std::to_string(i) + " joins two ghost elements";
        if (eL == eR && fL == fR) return "face " + std::to_string(i) + " connects a face to itself";
        // only owned elements get connectivity: ghosts are read, never computed
        std::string err = eL < nowned ? add_side(eL, fL, eR, fR, oL, oR, 1) : std::string();
        if (!err.empty()) return err;
        err = eR < nowned ? add_side(eR, fR, eL, fL, oR, oL, 0) : std::string();
        if (!err.empty()) return err;
    }
    for (int e = 0; e < nowned; ++e)
        for (int f = 0; f < 6; ++f)
            if (out.conn[(static_cast<size_t>(e) * 6 + f) * 2] < 0)
                return "unsupported: face " + std::to_string(f) + " of element " + std::to_string(e) +
                       " is a boundary face (only periodic meshes are handled)";
    out.ncodes = static_cast<int>(code_of.size());
    if (out.general) general_face_normals(mv, m, canon_inv, order_inv, out);
    return "";
}

}  // namespace dgh
