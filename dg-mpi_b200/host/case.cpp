// case.cpp -- see case.h.
#include "case.h"

#include <cmath>

#include "../csrc/dg_physics.cuh"

namespace dgh {

void project_initial_condition(const PreparedMesh& pm, const Tables1D& t, int ic_type, const double* data,
                               double gamma, double R, double time, double* Uc, int e_begin, int e_end)
{
    const int n = t.n, me = t.me, nb = n * n * n;
    const int ne = e_end < 0 ? pm.ne : e_end;
#pragma omp parallel
    {
        std::vector<double> f(static_cast<size_t>(me) * me * me * kNS);
        std::vector<double> t1(static_cast<size_t>(kNS) * me * me * n), t2(static_cast<size_t>(kNS) * me * n * n),
            r(static_cast<size_t>(kNS) * nb), r2(static_cast<size_t>(kNS) * nb);
#pragma omp for schedule(static)
        for (int e = e_begin; e < ne; ++e) {
            const GeoClass& g = pm.classes[pm.geo_class[e]];
            const double* X0 = &pm.X0[static_cast<size_t>(e) * 3];
            // f(q) * w_q * djac at the over-integration points
            for (int k = 0; k < me; ++k)
                for (int j = 0; j < me; ++j)
                    for (int i = 0; i < me; ++i) {
                        const double xi[3] = {t.xe[i] + 1.0, t.xe[j] + 1.0, t.xe[k] + 1.0};
                        double x[3];
                        for (int a = 0; a < 3; ++a)
                            x[a] = X0[a] + g.J[a * 3 + 0] * xi[0] + g.J[a * 3 + 1] * xi[1] + g.J[a * 3 + 2] * xi[2];
                        double U[kNS];
                        dgp::initial_state(ic_type, data, gamma, R, x, time, U);
                        const double cw = (t.we[i] * t.we[j]) * t.we[k] * g.djac;
                        const size_t q = (static_cast<size_t>(k) * me + j) * me + i;
                        for (int s = 0; s < kNS; ++s) f[q * kNS + s] = U[s] * cw;
                    }
            // rhs = (Be x Be x Be)^T f, contracted x, then y, then z
            for (int s = 0; s < kNS; ++s)
                for (int k = 0; k < me; ++k)
                    for (int j = 0; j < me; ++j)
                        for (int bx = 0; bx < n; ++bx) {
                            double acc = 0.0;
                            for (int i = 0; i < me; ++i)
                                acc += t.Be[i * n + bx] * f[((static_cast<size_t>(k) * me + j) * me + i) * kNS + s];
                            t1[((static_cast<size_t>(s) * me + k) * me + j) * n + bx] = acc;
                        }
            for (int s = 0; s < kNS; ++s)
                for (int k = 0; k < me; ++k)
                    for (int by = 0; by < n; ++by)
                        for (int bx = 0; bx < n; ++bx) {
                            double acc = 0.0;
                            for (int j = 0; j < me; ++j)
                                acc += t.Be[j * n + by] * t1[((static_cast<size_t>(s) * me + k) * me + j) * n + bx];
                            t2[((static_cast<size_t>(s) * me + k) * n + by) * n + bx] = acc;
                        }
            for (int s = 0; s < kNS; ++s)
                for (int bz = 0; bz < n; ++bz)
                    for (int byx = 0; byx < n * n; ++byx) {
                        double acc = 0.0;
                        for (int k = 0; k < me; ++k)
                            acc += t.Be[k * n + bz] * t2[((static_cast<size_t>(s) * me + k) * n * n) + byx];
                        r[static_cast<size_t>(s) * nb + bz * n * n + byx] = acc;
                    }
            // U = Minv^(x3) rhs / djac
            for (int s = 0; s < kNS; ++s) {
                double* rs = &r[static_cast<size_t>(s) * nb];
                double* os = &r2[static_cast<size_t>(s) * nb];
                for (int bz = 0; bz < n; ++bz)
                    for (int by = 0; by < n; ++by)
                        for (int bx = 0; bx < n; ++bx) {
                            double acc = 0.0;
                            for (int k = 0; k < n; ++k) acc += t.Minv[bx * n + k] * rs[(bz * n + by) * n + k];
                            os[(bz * n + by) * n + bx] = acc;
                        }
                for (int bz = 0; bz < n; ++bz)
                    for (int by = 0; by < n; ++by)
                        for (int bx = 0; bx < n; ++bx) {
                            double acc = 0.0;
                            for (int k = 0; k < n; ++k) acc += t.Minv[by * n + k] * os[(bz * n + k) * n + bx];
                            rs[(bz * n + by) * n + bx] = acc;
                        }
                for (int bz = 0; bz < n; ++bz)
                    for (int by = 0; by < n; ++by)
                        for (int bx = 0; bx < n; ++bx) {
                            double acc = 0.0;
                            for (int k = 0; k < n; ++k) acc += t.Minv[bz * n + k] * rs[(k * n + by) * n + bx];
                            Uc[(static_cast<size_t>(e - e_begin) * nb + (bz * n + by) * n + bx) * kNS + s] =
                                acc * g.inv_djac;
                        }
            }
        }
    }
}

double range_volume(const PreparedMesh& pm, int e_begin, int e_end)
{
    double v = 0.0;
    for (int e = e_begin; e < e_end; ++e) v += 8.0 * pm.classes[pm.geo_class[e]].djac;
    return v;
}

double range_hmin(const PreparedMesh& pm, int e_begin, int e_end)
{
    double h = 1e300;
    if (pm.general) {
        for (int e = e_begin; e < e_end; ++e) h = std::fmin(h, pm.elem_h[e]);
        return h;
    }
    std::vector<char> seen(pm.classes.size(), 0);
    for (int e = e_begin; e < e_end; ++e) {
        const int k = pm.geo_class[e];
        if (seen[k]) continue;
        seen[k] = 1;
        const GeoClass& g = pm.classes[k];
        for (int a = 0; a < 3; ++a)
            h = std::fmin(h, 2.0 * std::sqrt(g.J[0 * 3 + a] * g.J[0 * 3 + a] + g.J[1 * 3 + a] * g.J[1 * 3 + a] +
                                             g.J[2 * 3 + a] * g.J[2 * 3 + a]));
    }
    return h;
}

double cfl_time_step(const PreparedMesh& pm, int p, double gamma, const double* Uc, double cfl, int e_begin, int e_end)
{
    const int nb = (p + 1) * (p + 1) * (p + 1);
    if (e_end < 0) e_end = pm.ne;
    const size_t n = static_cast<size_t>(e_end - e_begin) * nb;
    double smax = 0.0;
    bool bad = false;
#pragma omp parallel for reduction(max : smax) reduction(|| : bad)
    for (long long i = 0; i < static_cast<long long>(n); ++i) {
        const double* U = Uc + i * kNS;
        const double P = dgp::pressure(gamma, U);
        if (!(U[0] > 0.0) || !(P > 0.0)) {
            bad = true;
            continue;
        }
        const double s = dgp::max_wave_speed(gamma, U);
        smax = std::fmax(smax, s);
    }
    if (bad || !(smax > 0.0)) return -1.0;
    const double hmin = (e_begin == 0 && e_end == pm.ne) ? pm.hmin : range_hmin(pm, e_begin, e_end);
    return cfl * hmin / ((2.0 * p + 1.0) * smax);
}

}  // namespace dgh
