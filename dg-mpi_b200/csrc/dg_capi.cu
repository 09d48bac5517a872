// dg_capi.cu -- the C ABI of include/dg_b200.h: context management, table
// upload, the graph-captured RK4 loop, layout transposes and the FP64
// reductions (L2 error, kinetic energy).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../host/case.h"
#include "../host/partition.h"
#include "dg_ctx.cuh"
#include "dg_tc.cuh"

using dgk::GeoDev;
using dgk::StageArgs;

int dgk::stage_variants(int p, const StageVariant** out)
{
    switch (p) {
        case 0: return stage_variants_p0(out);
        case 1: return stage_variants_p1(out);
        case 2: return stage_variants_p2(out);
        case 3: return stage_variants_p3(out);
        case 4: return stage_variants_p4(out);
        case 5: return stage_variants_p5(out);
        default: *out = nullptr; return 0;
    }
}

bool dgk::tc_operator(int p, const double* B1, std::vector<uint16_t>& out)
{
    if (p != 3) return false;
    out.assign(TcCfg<3>::kOpBytes / sizeof(uint16_t), 0);
    tc_operator_table<3>(B1, out.data());
    return true;
}

int dgk::tc_face_stride(int p)
{
    const int n = 5 * (p + 2) * (p + 2);
    return (n + 3) / 4 * 4;  // FP32 elements: a multiple of 16 bytes
}

namespace {

// tables of the IC / error rule (2*max(p,1)+2 points) and of the volume rule,
// used by the reductions
constexpr int kMaxMe = 12;
__constant__ double cVB[dgk::kMaxP + 1][dgk::kTabB];
__constant__ double cVW[dgk::kMaxP + 1][dgk::kMaxP + 2];
__constant__ double cBe[dgk::kMaxP + 1][kMaxMe * (dgk::kMaxP + 1)];
__constant__ double cWe[dgk::kMaxP + 1][kMaxMe];
__constant__ double cXe[dgk::kMaxP + 1][kMaxMe];
__constant__ double cXq[dgk::kMaxP + 1][dgk::kMaxP + 2];
__constant__ double cMi[dgk::kMaxP + 1][(dgk::kMaxP + 1) * (dgk::kMaxP + 1)];

std::mutex g_table_mutex;
bool g_tables_loaded[64] = {};
thread_local std::string g_create_error;

}  // namespace

namespace dgi {

int fail(dg_ctx* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

int load_constant_tables(dg_ctx* c)
{
    std::lock_guard<std::mutex> lk(g_table_mutex);
    if (c->device >= 0 && c->device < 64 && g_tables_loaded[c->device]) return DG_OK;
    // the current device must be c->device: constant symbols are per device
    double B[dgk::kMaxP + 1][dgk::kTabB] = {}, Dm[dgk::kMaxP + 1][dgk::kTabB] = {};
    double W[dgk::kMaxP + 1][dgk::kMaxP + 2] = {}, Mi[dgk::kMaxP + 1][(dgk::kMaxP + 1) * (dgk::kMaxP + 1)] = {};
    double Be[dgk::kMaxP + 1][kMaxMe * (dgk::kMaxP + 1)] = {}, We[dgk::kMaxP + 1][kMaxMe] = {};
    double Xe[dgk::kMaxP + 1][kMaxMe] = {}, Xq[dgk::kMaxP + 1][dgk::kMaxP + 2] = {};
    for (int p = 0; p <= dgk::kMaxP; ++p) {
        const dgh::Tables1D t = dgh::make_tables(p);
        std::copy(t.B.begin(), t.B.end(), B[p]);
        std::copy(t.D.begin(), t.D.end(), Dm[p]);
        std::copy(t.wq.begin(), t.wq.end(), W[p]);
        std::copy(t.xq.begin(), t.xq.end(), Xq[p]);
        std::copy(t.Minv.begin(), t.Minv.end(), Mi[p]);
        std::copy(t.Be.begin(), t.Be.end(), Be[p]);
        std::copy(t.we.begin(), t.we.end(), We[p]);
        std::copy(t.xe.begin(), t.xe.end(), Xe[p]);
    }
    (void)Dm;
    DG_CUDA(c, cudaMemcpyToSymbol(cMi, Mi, sizeof(Mi)));
    DG_CUDA(c, cudaMemcpyToSymbol(cVB, B, sizeof(B)));
    DG_CUDA(c, cudaMemcpyToSymbol(cVW, W, sizeof(W)));
    DG_CUDA(c, cudaMemcpyToSymbol(cBe, Be, sizeof(Be)));
    DG_CUDA(c, cudaMemcpyToSymbol(cWe, We, sizeof(We)));
    DG_CUDA(c, cudaMemcpyToSymbol(cXe, Xe, sizeof(Xe)));
    DG_CUDA(c, cudaMemcpyToSymbol(cXq, Xq, sizeof(Xq)));
    if (c->device >= 0 && c->device < 64) g_tables_loaded[c->device] = true;
    return DG_OK;
}

// ---------------------------------------------------------------------------
// stage launches

bool variant_matches(const dg_ctx* c, int v)
{
    const dgk::StageVariant* vs = nullptr;
    const int nv = dgk::stage_variants(c->p, &vs);
    return v >= 0 && v < nv && (vs[v].fp32 != 0) == (c->precision == DG_PREC_MIXED_FP32) &&
           ((vs[v].flags & dgk::kGE) != 0) == c->pm.general && (!(vs[v].flags & dgk::kFX) || c->d_fflux) &&
           (!(vs[v].flags & dgk::kTC) || c->d_tcop);
}

// Sets the variant's shared-memory attribute and its persistent grid size
// (SM count x resident CTAs per SM, capped by the number of batches).
int prepare_variant(dg_ctx* c, int v)
{
    const dgk::StageVariant* vs = nullptr;
    const int nv = dgk::stage_variants(c->p, &vs);
    if (v < 0 || v >= nv || v >= kMaxVariants) return fail(c, DG_ERR_ARG, "stage variant index out of range");
    if (c->variant_grid[v] > 0) return DG_OK;
    const dgk::StageVariant& sv = vs[v];
    DG_CUDA(c, cudaFuncSetAttribute(sv.func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sv.smem));
    // the tensor-core kernel runs two ~100 KB CTAs per SM: ask for the largest
    // shared-memory carveout (otherwise the occupancy query, and the launch,
    // may settle for one)
    if (sv.flags & dgk::kTC)
        DG_CUDA(c, cudaFuncSetAttribute(sv.func, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
    int dev_sms = 0, per_sm = 0;
    DG_CUDA(c, cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device));
    DG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sv.func, sv.NT, sv.smem));
    if (per_sm < 1) return fail(c, DG_ERR_UNSUPPORTED, "stage kernel variant does not fit on an SM");
    // the tensor-core kernel is built for two resident CTAs per SM (registers
    // and shared memory sized for it; its CTAs never wait on one another, so a
    // CTA that finds no room simply starts later); the occupancy query has been
    // seen to report one for it
    if (sv.flags & dgk::kTC) per_sm = std::max(per_sm, 2);
    const int batches = (c->ne + sv.E - 1) / sv.E;
    if (sv.face_launch) {
        if (!c->d_fflux) return fail(c, DG_ERR_UNSUPPORTED, "face-kernel variant on a context without a face list");
        int face_per_sm = 0;
        DG_CUDA(c, cudaFuncSetAttribute(sv.face_func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sv.face_smem));
        DG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&face_per_sm, sv.face_func, sv.face_threads, sv.face_smem));
        if (face_per_sm < 1) return fail(c, DG_ERR_UNSUPPORTED, "face kernel does not fit on an SM");
        const int fb = sv.face_batch;
        c->variant_face_grid[v] = std::max(1, std::min((c->nface + fb - 1) / fb, dev_sms * face_per_sm));
    }
    c->variant_grid[v] = std::max(1, std::min(batches, dev_sms * per_sm));
    return DG_OK;
}

void stage_args(const dg_ctx* c, int mode, const double* Us, const double* U0, double* out, double dt, int e_begin,
                int e_end, StageArgs& a)
{
    a = StageArgs{};
    a.Us = Us;
    a.U0 = U0;
    a.acc = c->d_acc;
    a.out = out;
    a.conn = c->d_conn;
    a.frec = c->d_frec;
    a.geo_class = c->d_geo_class;
    a.geo = c->d_geo;
    a.cmap = c->d_cmap;
    a.gjd = c->d_gjd;
    a.gnrm = c->d_gnrm;
    a.gimm = c->d_gimm;
    a.gfsd = c->d_gfsd;
    a.faces = c->d_faces;
    a.nface = c->nface;
    a.fflux = c->d_fflux;
    a.fstride = 5 * (c->p + 2) * (c->p + 2);
    a.tcop = c->d_tcop;
    a.status = c->d_status;
    a.e_begin = e_begin;
    a.ne = e_end;
    a.flux = c->flux;
    a.mode = mode;
    a.gamma = c->gamma;
    a.dt = dt;
    a.tab = c->stage_tab;
    const dgk::StageVariant* vs = nullptr;
    dgk::stage_variants(c->p, &vs);
    // the tensor-core kernel bulk-copies each face's fluxes: a 16-byte multiple per face
    if (vs[c->variant].flags & dgk::kTC) a.fstride = dgk::tc_face_stride(c->p);
}

int launch_stage(dg_ctx* c, int mode, const double* Us, const double* U0, double* out, double dt, int e_begin, int e_end)
{
    if (e_end < 0) e_end = c->ne;
    if (e_begin < 0 || e_end > c->ne || e_begin > e_end) return fail(c, DG_ERR_ARG, "stage element range out of bounds");
    if (e_begin == e_end) return DG_OK;
    StageArgs a;
    stage_args(c, mode, Us, U0, out, dt, e_begin, e_end, a);
    int rc = prepare_variant(c, c->variant);
    if (rc) return rc;
    const dgk::StageVariant* vs = nullptr;
    dgk::stage_variants(c->p, &vs);
    const dgk::StageVariant& sv = vs[c->variant];
    if (sv.face_launch) {
        // the fluxes of the faces this element range is the first to need (the
        // stage kernel reads them): all faces, the faces touching an interior
        // element, or the rest
        int f0 = 0, f1 = c->nface;
        if (e_begin == 0 && e_end == c->ninterior && e_end < c->ne) f1 = c->nface_inner;
        else if (e_begin == c->ninterior && e_begin > 0 && e_end == c->ne) f0 = c->nface_inner;
        else if (e_begin != 0 || e_end != c->ne) return fail(c, DG_ERR_ARG, "face-kernel variant on an element range");
        a.face_begin = f0;
        a.nface = f1;
        const int fb = sv.face_batch;
        if (f1 > f0) DG_CUDA(c, sv.face_launch(a, std::min(c->variant_face_grid[c->variant], (f1 - f0 + fb - 1) / fb), c->stream));
    }
    const int batches = (e_end - e_begin + sv.E - 1) / sv.E;
    DG_CUDA(c, sv.launch(a, std::min(c->variant_grid[c->variant], batches), c->stream));
    return DG_OK;
}

// ---------------------------------------------------------------------------
// layout transposes between the host layout [ne][nb][5] and the device
// layout [ne][5][nb]

__global__ void to_device_layout(const double* __restrict__ src, double* __restrict__ dst, long long n, int nb)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long e = i / (5LL * nb);
        const int r = (int)(i - e * 5LL * nb), v = r / nb, b = r - v * nb;
        dst[i] = src[(e * nb + b) * 5 + v];
    }
}

__global__ void to_host_layout(const double* __restrict__ src, double* __restrict__ dst, long long n, int nb)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long e = i / (5LL * nb);
        const int r = (int)(i - e * 5LL * nb), b = r / 5, v = r - b * 5;
        dst[i] = src[(e * 5 + v) * nb + b];
    }
}

// ---------------------------------------------------------------------------
// halo exchange: boundary slices [nslices][5][n*n] of the (element, face)
// pairs of the plan, gathered from owned elements / scattered into ghosts

__device__ __forceinline__ int slice_index_rt(int n, int f, int b0, int b1)
{
    const int ax = dgk::face_axis(f), sidx = dgk::face_side(f) ? n - 1 : 0;
    if (ax == 0) return b1 * n * n + b0 * n + sidx;
    if (ax == 1) return b1 * n * n + sidx * n + b0;
    return sidx * n * n + b1 * n + b0;
}

__global__ void halo_pack_kernel(const double* __restrict__ U, const int2* __restrict__ list, int nslices, int n,
                                 double* __restrict__ out)
{
    const int n2 = n * n, nb = n2 * n, per = 5 * n2;
    const long long total = (long long)nslices * per;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / per), r = (int)(i - (long long)s * per), v = r / n2, b = r - v * n2;
        const int2 ef = list[s];
        out[i] = U[((size_t)ef.x * 5 + v) * nb + slice_index_rt(n, ef.y, b % n, b / n)];
    }
}

__global__ void halo_unpack_kernel(double* __restrict__ U, const int2* __restrict__ list, int nslices, int n,
                                   const double* __restrict__ in)
{
    const int n2 = n * n, nb = n2 * n, per = 5 * n2;
    const long long total = (long long)nslices * per;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / per), r = (int)(i - (long long)s * per), v = r / n2, b = r - v * n2;
        const int2 ef = list[s];
        U[((size_t)ef.x * 5 + v) * nb + slice_index_rt(n, ef.y, b % n, b / n)] = in[i];
    }
}

// ---------------------------------------------------------------------------
// reductions: one CTA per element (grid-stride), threads over points; per-CTA
// partial sums land in a scratch array that the host adds in a fixed order.

// Position and det J at reference point xi of a trilinear element with nodes
// X [8][3] (the geometric basis of basis/tools.cpp:42-66; the same operations
// as the host's dgh::trilinear_jacobian).
__device__ void trilinear_point(const double* __restrict__ X, const double* xi, double* x, double* djac)
{
    double jac[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    x[0] = x[1] = x[2] = 0.0;
    for (int n = 0; n < 8; ++n) {
        double phi = 1.0, dphi[3];
        for (int j = 0; j < 3; ++j) {
            double g = 1.0;
            for (int a = 0; a < 3; ++a) {
                const double s = ((n >> a) & 1) ? 1.0 : -1.0;
                g *= a == j ? 0.5 * s : 0.5 * (1.0 + s * xi[a]);
            }
            dphi[j] = g;
            phi *= 0.5 * (1.0 + (((n >> j) & 1) ? 1.0 : -1.0) * xi[j]);
        }
        for (int i = 0; i < 3; ++i) {
            x[i] += phi * X[n * 3 + i];
            for (int j = 0; j < 3; ++j) jac[i * 3 + j] += X[n * 3 + i] * dphi[j];
        }
    }
    *djac = jac[0] * jac[4] * jac[8] - jac[0] * jac[5] * jac[7] - jac[1] * jac[3] * jac[8] + jac[1] * jac[5] * jac[6] +
            jac[2] * jac[3] * jac[7] - jac[2] * jac[4] * jac[6];
}

struct ReduceArgs {
    const double* U;        // device state [ne][5][nb]
    const int* geo_class;
    const GeoDev* geo;
    const double* X0;       // [ne][3]
    const double* J;        // [nclasses][9]
    const double* gnodes;   // general geometry: element nodes [ne][8][3] (else null)
    double* partials;       // [gridDim.x][5]
    int ne, ic_type, kind;  // kind 0: L2 error, 1: kinetic energy
    double gamma, R, t;
    double data[16];
};

template <int P>
__global__ void __launch_bounds__(256) reduce_kernel(ReduceArgs a)
{
    constexpr int N = P + 1, NB = N * N * N;
    __shared__ double sU[5 * NB];
    __shared__ double red[5][256];
    const int me = a.kind == 0 ? (P > 1 ? 2 * P + 2 : 4) : P + 2;
    const double* Bq = a.kind == 0 ? cBe[P] : cVB[P];
    const double* Wq = a.kind == 0 ? cWe[P] : cVW[P];
    const double* Xq = a.kind == 0 ? cXe[P] : cXq[P];
    double acc[5] = {0, 0, 0, 0, 0};
    for (int e = blockIdx.x; e < a.ne; e += gridDim.x) {
        __syncthreads();
        for (int i = threadIdx.x; i < 5 * NB; i += blockDim.x) sU[i] = a.U[(size_t)e * 5 * NB + i];
        __syncthreads();
        const int cls = a.geo_class[e];
        const double* J = a.J + cls * 9;
        const double djac = 1.0 / a.geo[cls].inv_djac;
        for (int q = threadIdx.x; q < me * me * me; q += blockDim.x) {
            const int i = q % me, j = (q / me) % me, k = q / (me * me);
            double Uq[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                double sz = 0.0;
                for (int bz = 0; bz < N; ++bz) {
                    double sy = 0.0;
                    for (int by = 0; by < N; ++by) {
                        double sx = 0.0;
#pragma unroll
                        for (int bx = 0; bx < N; ++bx) sx += Bq[i * N + bx] * sU[v * NB + (bz * N + by) * N + bx];
                        sy += Bq[j * N + by] * sx;
                    }
                    sz += Bq[k * N + bz] * sy;
                }
                Uq[v] = sz;
            }
            double x[3], dj = djac;
            if (a.gnodes) {
                const double xr[3] = {Xq[i], Xq[j], Xq[k]};
                trilinear_point(a.gnodes + (size_t)e * 24, xr, x, &dj);
            } else {
                const double xi[3] = {Xq[i] + 1.0, Xq[j] + 1.0, Xq[k] + 1.0};
                for (int d = 0; d < 3; ++d)
                    x[d] = a.X0[(size_t)e * 3 + d] + J[d * 3 + 0] * xi[0] + J[d * 3 + 1] * xi[1] + J[d * 3 + 2] * xi[2];
            }
            const double w = (Wq[i] * Wq[j]) * Wq[k] * dj;
            if (a.kind == 0) {
                double Ue[5];
                dgp::initial_state(a.ic_type, a.data, a.gamma, a.R, x, a.t, Ue);
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    const double d = Uq[v] - Ue[v];
                    acc[v] += d * d * w;
                }
            } else {
                acc[0] += 0.5 * (Uq[1] * Uq[1] + Uq[2] * Uq[2] + Uq[3] * Uq[3]) / Uq[0] * w;
            }
        }
    }
    __syncthreads();
    for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int v = 0; v < 5; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 5; ++v) a.partials[blockIdx.x * 5 + v] = red[v][0];
}

int run_reduce(dg_ctx* c, int kind, int ic_type, const double* data, int ndata, double t, double* out5, int e0, int ne,
               double gamma, double R)
{
    ReduceArgs a{};
    a.U = c->d_U0 + static_cast<size_t>(e0) * 5 * c->nb;
    a.geo_class = c->d_geo_class + e0;
    a.geo = c->d_geo;
    a.X0 = c->d_X0 + static_cast<size_t>(e0) * 3;
    a.gnodes = c->pm.general ? c->d_gnodes + static_cast<size_t>(e0) * 24 : nullptr;
    a.partials = c->d_partials;
    a.ne = ne;
    a.ic_type = ic_type;
    a.kind = kind;
    a.gamma = gamma;
    a.R = R;
    a.t = t;
    for (int i = 0; i < ndata && i < 16; ++i) a.data[i] = data[i];
    // per-class Jacobians, kept on the device after the classes
    a.J = reinterpret_cast<const double*>(c->d_geo + c->pm.classes.size());
    switch (c->p) {
        case 0: reduce_kernel<0><<<c->red_grid, 256, 0, c->stream>>>(a); break;
        case 1: reduce_kernel<1><<<c->red_grid, 256, 0, c->stream>>>(a); break;
        case 2: reduce_kernel<2><<<c->red_grid, 256, 0, c->stream>>>(a); break;
        case 3: reduce_kernel<3><<<c->red_grid, 256, 0, c->stream>>>(a); break;
        case 4: reduce_kernel<4><<<c->red_grid, 256, 0, c->stream>>>(a); break;
        case 5: reduce_kernel<5><<<c->red_grid, 256, 0, c->stream>>>(a); break;
        default: return fail(c, DG_ERR_UNSUPPORTED, "order out of range");
    }
    DG_CUDA(c, cudaGetLastError());
    std::vector<double> part(static_cast<size_t>(c->red_grid) * 5);
    DG_CUDA(c, cudaMemcpyAsync(part.data(), c->d_partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int v = 0; v < 5; ++v) out5[v] = 0.0;
    for (int b = 0; b < c->red_grid; ++b)
        for (int v = 0; v < 5; ++v) out5[v] += part[static_cast<size_t>(b) * 5 + v];
    return DG_OK;
}

// ---------------------------------------------------------------------------
// L2 projection of an initial condition on the device: the steps of
// dgh::project_initial_condition (Solver::init_state_from_fcn +
// SolverTools::L2_projection, src/solver/base.cpp:113-223,
// src/solver/tools.cpp:66-122) for affine elements, one CTA per element:
// f = U_ic(x_q) w_q det J at the 2*max(p,1)+2 point rule, rhs = (Be x Be x Be)^T f
// contracted x, y, z, then U = (Minv x Minv x Minv) rhs / det J.

struct ProjectArgs {
    double* U;              // device state [ne][5][nb]
    const int* geo_class;
    const GeoDev* geo;
    const double* X0;       // [ne][3]
    const double* J;        // [nclasses][9]
    // general geometry (else null): element nodes [ne][8][3] and the inverse
    // mass matrices, transposed [ne][nb][nb]
    const double* gnodes;
    const double* gimm;
    int e_begin, e_end, ic_type;
    double gamma, R, t;
    double data[16];
};

template <int P>
constexpr int project_points() { return P > 1 ? 2 * P + 2 : 4; }

template <int P>
constexpr size_t project_smem_bytes()
{
    constexpr int N = P + 1, ME = project_points<P>();
    return sizeof(double) * 5 * (ME * ME * ME + ME * ME * N + ME * N * N + N * N * N);
}

template <int P>
__global__ void __launch_bounds__(256) project_kernel(ProjectArgs a)
{
    constexpr int N = P + 1, NB = N * N * N, ME = project_points<P>(), Q = ME * ME * ME;
    extern __shared__ double psm[];
    double* f = psm;                     // [5][k][j][i]
    double* t1 = f + 5 * Q;              // [5][k][j][bx]
    double* t2 = t1 + 5 * ME * ME * N;   // [5][k][by][bx]
    double* r = t2 + 5 * ME * N * N;     // [5][bz][by][bx]
    const double* Be = cBe[P];
    const double* We = cWe[P];
    const double* Xe = cXe[P];
    const double* Mi = cMi[P];
    for (int e = a.e_begin + blockIdx.x; e < a.e_end; e += gridDim.x) {
        const int cls = a.geo_class[e];
        const double* J = a.J + cls * 9;
        const double inv_djac = a.geo[cls].inv_djac, djac = 1.0 / inv_djac;
        __syncthreads();
        for (int q = threadIdx.x; q < Q; q += blockDim.x) {
            const int i = q % ME, j = (q / ME) % ME, k = q / (ME * ME);
            double x[3], U[5], dj = djac;
            if (a.gnodes) {
                const double xr[3] = {Xe[i], Xe[j], Xe[k]};
                trilinear_point(a.gnodes + (size_t)e * 24, xr, x, &dj);
            } else {
                const double xi[3] = {Xe[i] + 1.0, Xe[j] + 1.0, Xe[k] + 1.0};
                for (int d = 0; d < 3; ++d)
                    x[d] = a.X0[(size_t)e * 3 + d] + J[d * 3 + 0] * xi[0] + J[d * 3 + 1] * xi[1] + J[d * 3 + 2] * xi[2];
            }
            dgp::initial_state(a.ic_type, a.data, a.gamma, a.R, x, a.t, U);
            const double cw = (We[i] * We[j]) * We[k] * dj;
#pragma unroll
            for (int v = 0; v < 5; ++v) f[v * Q + q] = U[v] * cw;
        }
        __syncthreads();
        for (int o = threadIdx.x; o < 5 * ME * ME * N; o += blockDim.x) {  // x
            const int bx = o % N, kj = o / N;  // kj = (v*ME + k)*ME + j
            double acc = 0.0;
            for (int i = 0; i < ME; ++i) acc += Be[i * N + bx] * f[kj * ME + i];
            t1[o] = acc;
        }
        __syncthreads();
        for (int o = threadIdx.x; o < 5 * ME * N * N; o += blockDim.x) {  // y
            const int bx = o % N, by = (o / N) % N, vk = o / (N * N);
            double acc = 0.0;
            for (int j = 0; j < ME; ++j) acc += Be[j * N + by] * t1[(vk * ME + j) * N + bx];
            t2[o] = acc;
        }
        __syncthreads();
        for (int o = threadIdx.x; o < 5 * NB; o += blockDim.x) {  // z
            const int byx = o % (N * N), bz = (o / (N * N)) % N, v = o / NB;
            double acc = 0.0;
            for (int k = 0; k < ME; ++k) acc += Be[k * N + bz] * t2[((v * ME + k) * N * N) + byx];
            r[o] = acc;
        }
        __syncthreads();
        if (a.gimm) {  // the element's dense inverse mass matrix
            for (int o = threadIdx.x; o < 5 * NB; o += blockDim.x) {
                const int j = o % NB, v = o / NB;
                const double* im = a.gimm + (size_t)e * NB * NB + j;
                double acc = 0.0;
                for (int k = 0; k < NB; ++k) acc += im[(size_t)k * NB] * r[v * NB + k];
                a.U[(size_t)e * 5 * NB + o] = acc;
            }
            continue;
        }
        for (int o = threadIdx.x; o < 5 * NB; o += blockDim.x) {  // Minv along x, into t2
            const int bx = o % N, row = o / N;
            double acc = 0.0;
            for (int k = 0; k < N; ++k) acc += Mi[bx * N + k] * r[row * N + k];
            t2[o] = acc;
        }
        __syncthreads();
        for (int o = threadIdx.x; o < 5 * NB; o += blockDim.x) {  // along y, into r
            const int bx = o % N, by = (o / N) % N, vz = o / (N * N);
            double acc = 0.0;
            for (int k = 0; k < N; ++k) acc += Mi[by * N + k] * t2[(vz * N + k) * N + bx];
            r[o] = acc;
        }
        __syncthreads();
        for (int o = threadIdx.x; o < 5 * NB; o += blockDim.x) {  // along z, / det J
            const int byx = o % (N * N), bz = (o / (N * N)) % N, v = o / NB;
            double acc = 0.0;
            for (int k = 0; k < N; ++k) acc += Mi[bz * N + k] * r[(v * N + k) * N * N + byx];
            a.U[(size_t)e * 5 * NB + o] = acc * inv_djac;
        }
    }
}

template <int P>
int launch_project(dg_ctx* c, const ProjectArgs& a)
{
    constexpr size_t smem = project_smem_bytes<P>();
    DG_CUDA(c, cudaFuncSetAttribute(project_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int n = a.e_end - a.e_begin;
    int dev_sms = 0;
    DG_CUDA(c, cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device));
    const int grid = std::max(1, std::min(n, 8 * dev_sms));
    project_kernel<P><<<grid, 256, smem, c->stream>>>(a);
    DG_CUDA(c, cudaGetLastError());
    return DG_OK;
}

int project_ic_device(dg_ctx* c, int ic_type, const double* data, int ndata, double t, double gamma, double R, int e0,
                      int ne)
{
    if (ne <= 0) return DG_OK;
    ProjectArgs a{};
    a.U = c->d_U0;
    a.geo_class = c->d_geo_class;
    a.geo = c->d_geo;
    a.X0 = c->d_X0;
    a.J = reinterpret_cast<const double*>(c->d_geo + c->pm.classes.size());
    a.gnodes = c->pm.general ? c->d_gnodes : nullptr;
    a.gimm = c->pm.general ? c->d_gimm : nullptr;
    a.e_begin = e0;
    a.e_end = e0 + ne;
    a.ic_type = ic_type;
    a.gamma = gamma;
    a.R = R;
    a.t = t;
    for (int i = 0; i < ndata && i < 16; ++i) a.data[i] = data[i];
    switch (c->p) {
        case 0: return launch_project<0>(c, a);
        case 1: return launch_project<1>(c, a);
        case 2: return launch_project<2>(c, a);
        case 3: return launch_project<3>(c, a);
        case 4: return launch_project<4>(c, a);
        case 5: return launch_project<5>(c, a);
        default: return fail(c, DG_ERR_UNSUPPORTED, "order out of range");
    }
}

// ---------------------------------------------------------------------------
// allocation-free kinetic energy: the same per-element quadrature as
// reduce_kernel (kind 1), with the per-block partial sums in a static device
// array instead of context memory, and a one-block finalisation on the device

constexpr int kNoAllocElemsPerBlock = 64;
constexpr int kNoAllocMaxBlocks = 16384;  // two doubles each: 32768 doubles, 256 KB
constexpr long long kNoAllocMaxElems = 1LL * kNoAllocElemsPerBlock * kNoAllocMaxBlocks;

static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxBlocks];

std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[64] = {};

template <int P>
__global__ void __launch_bounds__(256) ke_partials_noalloc(const double* __restrict__ U, const double* __restrict__ djac,
                                                           int ne, double* __restrict__ scratch)
{
    constexpr int N = P + 1, NB = N * N * N, M = P + 2;
    __shared__ double sU[5 * NB];
    __shared__ double red[2][256];
    const double* Bq = cVB[P];
    const double* Wq = cVW[P];
    double ke = 0.0, vol = 0.0;
    const int e_begin = blockIdx.x * kNoAllocElemsPerBlock;
    const int e_end = min(ne, e_begin + kNoAllocElemsPerBlock);
    for (int e = e_begin; e < e_end; ++e) {
        __syncthreads();
        for (int i = threadIdx.x; i < 5 * NB; i += blockDim.x) sU[i] = U[(size_t)e * 5 * NB + i];
        __syncthreads();
        const double dj = djac[e];
        for (int q = threadIdx.x; q < M * M * M; q += blockDim.x) {
            const int i = q % M, j = (q / M) % M, k = q / (M * M);
            double Uq[4];
            for (int v = 0; v < 4; ++v) {
                double sz = 0.0;
                for (int bz = 0; bz < N; ++bz) {
                    double sy = 0.0;
                    for (int by = 0; by < N; ++by) {
                        double sx = 0.0;
                        for (int bx = 0; bx < N; ++bx) sx += Bq[i * N + bx] * sU[v * NB + (bz * N + by) * N + bx];
                        sy += Bq[j * N + by] * sx;
                    }
                    sz += Bq[k * N + bz] * sy;
                }
                Uq[v] = sz;
            }
            const double w = (Wq[i] * Wq[j]) * Wq[k] * dj;
            ke += 0.5 * (Uq[1] * Uq[1] + Uq[2] * Uq[2] + Uq[3] * Uq[3]) / Uq[0] * w;
            vol += w;
        }
    }
    red[0][threadIdx.x] = ke;
    red[1][threadIdx.x] = vol;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[2 * blockIdx.x] = red[0][0];
        scratch[2 * blockIdx.x + 1] = red[1][0];
    }
}

// sums the nblocks partials in a fixed order (deterministic) and writes KE / V
__global__ void __launch_bounds__(256) ke_finalize_noalloc(const double* __restrict__ scratch, int nblocks,
                                                           double* __restrict__ out)
{
    __shared__ double red[2][256];
    double ke = 0.0, vol = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        ke += scratch[2 * b];
        vol += scratch[2 * b + 1];
    }
    red[0][threadIdx.x] = ke;
    red[1][threadIdx.x] = vol;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0][0] / red[1][0];
}

int check_status(dg_ctx* c)
{
    unsigned st = 0;
    DG_CUDA(c, cudaMemcpyAsync(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (st) {
        c->status_accum |= st;
        DG_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
        DG_CUDA(c, cudaStreamSynchronize(c->stream));
        char buf[160];
        if (st & dgk::kStatusTimeout) {
            snprintf(buf, sizeof(buf), "a bounded device wait gave up (status 0x%x)", st);
            return fail(c, DG_ERR_TIMEOUT, buf);
        }
        snprintf(buf, sizeof(buf), "non-physical state detected on the device (status 0x%x)", st);
        return fail(c, DG_ERR_NONPHYSICAL, buf);
    }
    return DG_OK;
}

int upload_range(dg_ctx* c, const double* Uc, double* dst, int e0, int ne)
{
    const size_t n = static_cast<size_t>(ne) * c->nb * 5, off = static_cast<size_t>(e0) * c->nb * 5;
    if (n == 0) return DG_OK;
    DG_CUDA(c, cudaMemcpyAsync(c->d_out + off, Uc, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    to_device_layout<<<1024, 256, 0, c->stream>>>(c->d_out + off, dst + off, (long long)n, c->nb);
    DG_CUDA(c, cudaGetLastError());
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int download_range(dg_ctx* c, const double* src, double* Uc, int e0, int ne)
{
    const size_t n = static_cast<size_t>(ne) * c->nb * 5, off = static_cast<size_t>(e0) * c->nb * 5;
    if (n == 0) return DG_OK;
    double* stage = (c->d_acc == src ? c->d_out : c->d_Ub) + off;
    to_host_layout<<<1024, 256, 0, c->stream>>>(src + off, stage, (long long)n, c->nb);
    DG_CUDA(c, cudaGetLastError());
    DG_CUDA(c, cudaMemcpyAsync(Uc, stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int upload_state_host_layout(dg_ctx* c, const double* Uc, double* dst) { return upload_range(c, Uc, dst, 0, c->ne); }
int download_host_layout(dg_ctx* c, const double* src, double* Uc) { return download_range(c, src, Uc, 0, c->ne); }

double energy_reference(const dg_ctx* c, const double* Uc, int ne)
{
    if (c->precision != DG_PREC_MIXED_FP32 || ne <= 0) return 0.0;
    const long long n = 1LL * ne * c->nb;
    // fixed blocks summed in order: the same state gives the same bits for any
    // thread count (a batch case and a context of that case must agree exactly)
    constexpr int kBlocks = 256;
    double part[kBlocks];
#pragma omp parallel for schedule(static)
    for (int b = 0; b < kBlocks; ++b) {
        const long long i0 = n * b / kBlocks, i1 = n * (b + 1) / kBlocks;
        double s = 0.0;
        for (long long i = i0; i < i1; ++i) s += Uc[i * 5 + 4];
        part[b] = s;
    }
    double sum = 0.0;
    for (int b = 0; b < kBlocks; ++b) sum += part[b];
    const double m = sum / static_cast<double>(n);
    return std::isfinite(m) ? m : 0.0;
}

int upload_geometry(dg_ctx* c, cudaStream_t s)
{
    // geometry classes, followed by their Jacobians (used by the reductions)
    const size_t ncls = c->pm.classes.size();
    std::vector<unsigned char> blob(ncls * (sizeof(GeoDev) + 9 * sizeof(double)));
    for (size_t k = 0; k < ncls; ++k) {
        GeoDev g{};
        const auto& src = c->pm.classes[k];
        std::memcpy(g.JD, src.JD, sizeof(g.JD));
        g.inv_djac = src.inv_djac;
        g.dtf = c->class_dtf[k];
        g.eref = c->class_eref[k];
        std::memcpy(g.N, src.N, sizeof(g.N));
        std::memcpy(g.nmag, src.nmag, sizeof(g.nmag));
        std::memcpy(g.nhat, src.nhat, sizeof(g.nhat));
        std::memcpy(g.nunit, src.nunit, sizeof(g.nunit));
        std::memcpy(blob.data() + k * sizeof(GeoDev), &g, sizeof(GeoDev));
        std::memcpy(blob.data() + ncls * sizeof(GeoDev) + k * 9 * sizeof(double), src.J, 9 * sizeof(double));
    }
    DG_CUDA(c, cudaMemcpyAsync(c->d_geo, blob.data(), blob.size(), cudaMemcpyHostToDevice, s));
    DG_CUDA(c, cudaStreamSynchronize(s));
    return DG_OK;
}

// The FP64 residual of the uniform state (1, 0, 0, 0, 1/(gamma-1)) -- at rest,
// unit pressure -- into d_gfsd, with the first FP64 general-geometry variant
// (see dgk::StageArgs::gfsd); d_U0 is left zeroed.
int unit_pressure_residual(dg_ctx* c)
{
    const int nv = dg_num_stage_variants(c->p);
    const dgk::StageVariant* vs = nullptr;
    dgk::stage_variants(c->p, &vs);
    int v64 = -1;
    for (int v = 0; v < nv && v64 < 0; ++v)
        if (!vs[v].fp32 && (vs[v].flags & dgk::kGE)) v64 = v;
    if (v64 < 0) return fail(c, DG_ERR_UNSUPPORTED, "no FP64 general-geometry stage kernel for this order");
    const size_t nstate = static_cast<size_t>(c->ne) * c->nb * 5;
    std::vector<double> U(nstate, 0.0);
    for (size_t e = 0; e < static_cast<size_t>(c->ne); ++e)
        for (int b = 0; b < c->nb; ++b) {
            U[(e * 5 + 0) * c->nb + b] = 1.0;
            U[(e * 5 + 4) * c->nb + b] = 1.0 / (c->gamma - 1.0);
        }
    DG_CUDA(c, cudaMemcpy(c->d_U0, U.data(), nstate * sizeof(double), cudaMemcpyHostToDevice));
    const int keep = c->variant;
    c->variant = v64;
    int rc = launch_stage(c, dgk::kModeResidual, c->d_U0, c->d_U0, c->d_gfsd, 0.0);
    c->variant = keep;
    if (rc) return rc;
    if ((rc = check_status(c)) != DG_OK) return rc;
    DG_CUDA(c, cudaMemsetAsync(c->d_U0, 0, nstate * sizeof(double), c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

void release(dg_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    cudaFree(c->d_U0); cudaFree(c->d_Ua); cudaFree(c->d_Ub); cudaFree(c->d_acc); cudaFree(c->d_out);
    cudaFree(c->d_conn); cudaFree(c->d_frec); cudaFree(c->d_geo_class); cudaFree(c->d_geo); cudaFree(c->d_cmap);
    cudaFree(c->d_X0); cudaFree(c->d_partials); cudaFree(c->d_status);
    cudaFree(c->d_gjd); cudaFree(c->d_gnrm); cudaFree(c->d_gimm); cudaFree(c->d_gnodes); cudaFree(c->d_gfsd);
    cudaFree(c->d_faces); cudaFree(c->d_fflux); cudaFree(c->d_tcop);
    cudaFree(c->d_halo_send); cudaFree(c->d_halo_recv);
    for (cudaEvent_t e : c->chunk_ev) cudaEventDestroy(e);
    c->chunk_ev.clear();
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->stream) cudaStreamDestroy(c->stream);
}

}  // namespace dgi

using namespace dgi;

int dgi::create_ctx(const dg_case_desc* cd, const dg_mesh_desc* md, const int* elem_tag, const dg_part_desc* part,
                    dg_ctx** out)
{
    g_create_error.clear();
    if (!cd || !md || !out) return fail(nullptr, DG_ERR_ARG, "dg_create: null argument");
    *out = nullptr;
    if (cd->order < 0 || cd->order > dgk::kMaxP) return fail(nullptr, DG_ERR_UNSUPPORTED, "order must be 0..5");
    if (cd->flux != DG_FLUX_LAX_FRIEDRICHS && cd->flux != DG_FLUX_HLLC) return fail(nullptr, DG_ERR_ARG, "unknown flux");
    if (!(cd->gamma > 1.0)) return fail(nullptr, DG_ERR_ARG, "gamma must exceed 1");
    if (cd->precision != DG_PREC_FP64 && cd->precision != DG_PREC_MIXED_FP32)
        return fail(nullptr, DG_ERR_ARG, "unknown precision mode");

    dg_ctx* c = new (std::nothrow) dg_ctx();
    if (!c) return fail(nullptr, DG_ERR_NOMEM, "host allocation failed");
    c->device = cd->device;
    c->p = cd->order;
    c->nb = (c->p + 1) * (c->p + 1) * (c->p + 1);
    c->flux = cd->flux;
    c->gamma = cd->gamma;
    c->R = cd->gas_constant;
    c->precision = cd->precision;

    dgh::MeshView mv;
    mv.nnode = md->nnode;
    mv.nelem = md->nelem;
    mv.nface = md->nface;
    mv.rank = md->rank;
    mv.coords = md->node_coords;
    mv.e2n = md->elem_to_node_ids;
    mv.faces = md->interior_faces;
    mv.tag = elem_tag;
    std::vector<int> elem_rank;
    dgh::HaloPlan plan;
    std::string perr;
    if (part) {
        const int ng = md->nelem - part->nowned;
        if (part->nowned < 1 || ng < 0 || part->ninterior < 0 || part->ninterior > part->nowned ||
            (ng > 0 && (!part->ghost_rank || !part->ghost_elem)))
            perr = "partition description out of range";
        for (int g = 0; perr.empty() && g < ng; ++g)
            if (part->ghost_rank[g] < 0 || part->ghost_elem[g] < 0) perr = "ghost " + std::to_string(g) + " has no owner";
        if (perr.empty()) {
            elem_rank.assign(md->nelem, md->rank);
            for (int g = 0; g < ng; ++g) elem_rank[part->nowned + g] = part->ghost_rank[g];
            mv.nowned = part->nowned;
            mv.elem_rank = elem_rank.data();
        }
    }
    try {
        if (perr.empty()) perr = dgh::prepare_mesh(mv, c->p + 2, c->pm);
        if (perr.empty() && part) perr = dgh::make_halo_plan(mv, part->ghost_elem, plan);
        c->tab = dgh::make_tables(c->p);
    } catch (const std::exception& ex) {
        perr = std::string("mesh preparation failed: ") + ex.what();
    }
    if (perr.empty() && part && c->pm.general)
        perr = "unsupported: non-affine elements in a partitioned context (general geometry runs unpartitioned)";
    if (perr.empty() && part) {
        // the interior elements must not read a ghost: they run while the exchange is in flight
        for (int e = 0; e < part->ninterior && perr.empty(); ++e)
            for (int f = 0; f < 6; ++f)
                if (c->pm.conn[(static_cast<size_t>(e) * 6 + f) * 2] >= part->nowned)
                    perr = "element " + std::to_string(e) + " is counted as interior but has a ghost neighbour";
    }
    if (!perr.empty()) {
        delete c;
        const bool unsup = perr.rfind("unsupported:", 0) == 0;
        return fail(nullptr, unsup ? DG_ERR_UNSUPPORTED : DG_ERR_ARG, perr);
    }
    c->ne = c->pm.nowned;
    c->ne_alloc = c->pm.ne;
    c->ninterior = part ? part->ninterior : 0;
    c->nslices = static_cast<int>(plan.send_elem.size());
    c->peer_rank = plan.peer_rank;
    c->peer_offset = plan.peer_offset;
    c->peer_count = plan.peer_count;
    std::copy(c->tab.B.begin(), c->tab.B.end(), c->stage_tab.B);
    std::copy(c->tab.D.begin(), c->tab.D.end(), c->stage_tab.D);
    std::copy(c->tab.wq.begin(), c->tab.wq.end(), c->stage_tab.W);
    std::copy(c->tab.Minv.begin(), c->tab.Minv.end(), c->stage_tab.Minv);
    for (size_t i = 0; i < c->tab.B.size(); ++i) c->stage_tab.Bf[i] = static_cast<float>(c->tab.B[i]);
    for (size_t i = 0; i < c->tab.D.size(); ++i) c->stage_tab.Df[i] = static_cast<float>(c->tab.D[i]);
    for (size_t i = 0; i < c->tab.wq.size(); ++i) c->stage_tab.Wf[i] = static_cast<float>(c->tab.wq[i]);
    {   // nodal derivative of the 1D basis: Dn[i*n + j] = l_j'(xi_i) at the equidistant nodes
        const int n = c->p + 1;
        const std::vector<double> xn = dgh::equidistant_nodes(n);
        std::vector<double> val(n), grad(n);
        for (int i = 0; i < n; ++i) {
            dgh::lagrange_1d(xn[i], xn, val.data(), grad.data());
            for (int j = 0; j < n; ++j) c->stage_tab.Dn[i * n + j] = static_cast<float>(grad[j]);
        }
    }
    {   // default launch variant: the first one compiled for the requested precision and geometry kind
        const int nv = dg_num_stage_variants(c->p);
        c->variant = -1;
        for (int v = 0; v < nv && c->variant < 0; ++v)
            if (variant_matches(c, v)) c->variant = v;
        if (c->variant < 0) {
            delete c;
            return fail(nullptr, DG_ERR_UNSUPPORTED, "no stage kernel compiled for this order, precision and geometry");
        }
    }
    // general geometry: the dense inverse mass matrix of every element (host,
    // once; nb^2 doubles per element) and the flux's normal data per face point
    std::vector<double> gimm, gnrm;
    if (c->pm.general) {
        const int nb = c->nb, nf = (c->p + 2) * (c->p + 2);
        gimm.resize(static_cast<size_t>(c->ne) * nb * nb);
        int singular = -1;
#pragma omp parallel for schedule(dynamic, 16)
        for (int e = 0; e < c->ne; ++e)
            if (!dgh::general_inverse_mass(c->tab, &c->pm.gnodes[static_cast<size_t>(e) * 24],
                                           &gimm[static_cast<size_t>(e) * nb * nb])) {
#pragma omp critical
                singular = e;
            }
        if (singular >= 0) {
            delete c;
            return fail(nullptr, DG_ERR_ARG, "element " + std::to_string(singular) + " has a singular mass matrix");
        }
        // per face point: n (N/|N| for Lax-Friedrichs, N * (1/|N|) for HLLC, as
        // in FaceRec), then |N| -- base/functions.cpp:40-49, euler/functions.cpp:309-311
        gnrm.resize(static_cast<size_t>(c->ne) * 6 * 4 * nf);
        for (size_t ef = 0; ef < static_cast<size_t>(c->ne) * 6; ++ef)
            for (int q = 0; q < nf; ++q) {
                const double* N = &c->pm.gN[ef * 3 * nf + q];
                const double N0 = N[0], N1 = N[nf], N2 = N[2 * nf];
                const double nm = std::sqrt(N0 * N0 + N1 * N1 + N2 * N2), inv = 1. / nm;
                double* o = &gnrm[ef * 4 * nf + q];
                if (c->flux == DG_FLUX_HLLC) {
                    o[0] = N0 * inv;
                    o[nf] = N1 * inv;
                    o[2 * nf] = N2 * inv;
                } else {
                    o[0] = N0 / nm;
                    o[nf] = N1 / nm;
                    o[2 * nf] = N2 / nm;
                }
                o[3 * nf] = nm;
            }
    }

    // the mesh is valid; now the device
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        delete c;
        return fail(nullptr, DG_ERR_CUDA, "no CUDA device available");
    }
    if (cd->device < 0 || cd->device >= ndev) {
        delete c;
        return fail(nullptr, DG_ERR_ARG, "device ordinal out of range");
    }

    int rc = DG_OK;
    auto bail = [&](int code) {
        g_create_error = c->err;
        release(c);
        delete c;
        return code;
    };
    if (cudaSetDevice(c->device) != cudaSuccess) {
        c->err = "cudaSetDevice failed";
        return bail(DG_ERR_CUDA);
    }
    if ((rc = load_constant_tables(c)) != DG_OK) return bail(rc);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        c->err = "cudaStreamCreate failed";
        return bail(DG_ERR_CUDA);
    }
    const size_t nstate = static_cast<size_t>(c->ne_alloc) * c->nb * 5;
    const size_t ncls = c->pm.classes.size();
    int dev_sms = 0;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    c->red_grid = std::max(1, std::min(c->ne, 4 * dev_sms));
    struct Alloc { void** p; size_t bytes; } allocs[] = {
        {(void**)&c->d_U0, nstate * sizeof(double)},
        {(void**)&c->d_Ua, nstate * sizeof(double)},
        {(void**)&c->d_Ub, nstate * sizeof(double)},
        {(void**)&c->d_acc, nstate * sizeof(double)},
        {(void**)&c->d_out, nstate * sizeof(double)},
        {(void**)&c->d_conn, static_cast<size_t>(c->ne_alloc) * 6 * sizeof(int2)},
        {(void**)&c->d_frec, static_cast<size_t>(std::max(1, c->ne)) * 6 * sizeof(dgk::FaceRec)},
        {(void**)&c->d_geo_class, static_cast<size_t>(c->ne_alloc) * sizeof(int)},
        {(void**)&c->d_geo, ncls * (sizeof(GeoDev) + 9 * sizeof(double))},
        {(void**)&c->d_cmap, std::max<size_t>(1, c->pm.cmap.size())},
        {(void**)&c->d_X0, static_cast<size_t>(c->ne_alloc) * 3 * sizeof(double)},
        {(void**)&c->d_halo_send, std::max<size_t>(1, c->nslices) * sizeof(int2)},
        {(void**)&c->d_halo_recv, std::max<size_t>(1, c->nslices) * sizeof(int2)},
        {(void**)&c->d_partials, static_cast<size_t>(c->red_grid) * 5 * sizeof(double)},
        {(void**)&c->d_status, sizeof(unsigned)},
        {(void**)&c->d_gjd, std::max<size_t>(1, c->pm.gjd.size()) * sizeof(double)},
        {(void**)&c->d_gnrm, std::max<size_t>(1, gnrm.size()) * sizeof(double)},
        {(void**)&c->d_gimm, std::max<size_t>(1, gimm.size()) * sizeof(double)},
        {(void**)&c->d_gnodes, std::max<size_t>(1, c->pm.gnodes.size()) * sizeof(double)},
        {(void**)&c->d_gfsd, (c->pm.general && c->precision == DG_PREC_MIXED_FP32 ? nstate : 1) * sizeof(double)},
    };
    for (auto& al : allocs) {
        if (cudaMalloc(al.p, al.bytes) != cudaSuccess) {
            cudaGetLastError();
            c->err = "device allocation of " + std::to_string(al.bytes) + " bytes failed";
            return bail(DG_ERR_NOMEM);
        }
    }
    std::vector<int2> conn(static_cast<size_t>(c->ne_alloc) * 6);
    for (size_t i = 0; i < conn.size(); ++i) conn[i] = make_int2(c->pm.conn[i * 2], c->pm.conn[i * 2 + 1]);
    // the face records of the owned elements (see dgk::FaceRec)
    std::vector<dgk::FaceRec> frec(static_cast<size_t>(std::max(1, c->ne)) * 6);
    for (int e = 0; e < c->ne; ++e)
        for (int f = 0; f < 6; ++f) {
            const int nbr = c->pm.conn[(static_cast<size_t>(e) * 6 + f) * 2];
            const int info = c->pm.conn[(static_cast<size_t>(e) * 6 + f) * 2 + 1];
            const int isL = (info >> 3) & 1, fn = info & 7;
            // the normal is the left element's (helpers.cpp:440-446)
            const dgh::GeoClass& gL = c->pm.classes[c->pm.geo_class[isL ? e : nbr]];
            const int fl = isL ? f : fn;
            dgk::FaceRec& r = frec[static_cast<size_t>(e) * 6 + f];
            for (int d = 0; d < 3; ++d) r.n[d] = c->flux == DG_FLUX_HLLC ? gL.nunit[fl][d] : gL.nhat[fl][d];
            r.nmag = gL.nmag[fl];
            r.nbr = nbr;
            r.info = info;
            r.cls = c->pm.geo_class[e];
            r.pad = -1;
        }
    // launch option FX: the face list.  A face between owned elements is
    // listed by its left side, a face next to a ghost by its owned side; the
    // faces touching an interior element come first (the interior range's
    // launch computes them while the halo exchange is in flight), the others
    // after.  Each owned side's record carries the face's number, with bit 30
    // set on the listed side (it reads the flux in its own point order).
    std::vector<int2> faces;
    const bool face_list = c->ne > 0;
    if (face_list) {
        auto rec = [&](int e, int f) -> dgk::FaceRec& { return frec[static_cast<size_t>(e) * 6 + f]; };
        auto listed = [&](int e, int f) {
            rec(e, f).pad = static_cast<int>(faces.size()) | (1 << 30);
            faces.push_back(make_int2(e, f));
        };
        for (int e = 0; e < c->ne; ++e)
            for (int f = 0; f < 6; ++f) {
                const dgk::FaceRec& r = rec(e, f);
                if (r.nbr < c->ne && ((r.info >> 3) & 1) && (e < c->ninterior || r.nbr < c->ninterior)) listed(e, f);
            }
        c->nface_inner = static_cast<int>(faces.size());
        if (c->ninterior == 0 && c->ne_alloc == c->ne) {
            // no ghosts: every face by its left side, ordered by the lower of
            // its two elements (stable in the left element and face)
            std::vector<std::array<int, 3>> order;
            for (int e = 0; e < c->ne; ++e)
                for (int f = 0; f < 6; ++f) {
                    const dgk::FaceRec& r = rec(e, f);
                    if (r.nbr < c->ne && ((r.info >> 3) & 1)) order.push_back({std::min(e, r.nbr), e, f});
                }
            std::stable_sort(order.begin(), order.end(),
                             [](const std::array<int, 3>& x, const std::array<int, 3>& y) { return x[0] < y[0]; });
            c->face_key.clear();
            for (const auto& o : order) {
                listed(o[1], o[2]);
                c->face_key.push_back(o[0]);
            }
        } else {
            for (int e = 0; e < c->ne; ++e)
                for (int f = 0; f < 6; ++f) {
                    const dgk::FaceRec& r = rec(e, f);
                    if (r.nbr >= c->ne || (((r.info >> 3) & 1) && e >= c->ninterior && r.nbr >= c->ninterior)) listed(e, f);
                }
        }
        for (int e = 0; e < c->ne; ++e)
            for (int f = 0; f < 6; ++f) {
                dgk::FaceRec& r = rec(e, f);
                if (r.nbr < c->ne && !((r.info >> 3) & 1)) r.pad = rec(r.nbr, r.info & 7).pad & 0x3fffffff;
            }
        c->nface = static_cast<int>(faces.size());
        // the face list and the flux buffer, when this order compiles a
        // face-kernel variant (a failed allocation leaves those variants out)
        const dgk::StageVariant* vs = nullptr;
        const int nv = dgk::stage_variants(c->p, &vs);
        bool has_fx = false;
        for (int v = 0; v < nv; ++v) has_fx = has_fx || (vs[v].flags & dgk::kFX);
        const size_t nflux = static_cast<size_t>(c->nface) * 5 * (c->p + 2) * (c->p + 2);
        if (has_fx && c->nface > 0) {
            if (cudaMalloc((void**)&c->d_faces, faces.size() * sizeof(int2)) != cudaSuccess ||
                cudaMalloc((void**)&c->d_fflux, nflux * sizeof(double)) != cudaSuccess ||
                cudaMemcpy(c->d_faces, faces.data(), faces.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess) {
                cudaGetLastError();
                cudaFree(c->d_faces);
                cudaFree(c->d_fflux);
                c->d_faces = nullptr;
                c->d_fflux = nullptr;
            }
        }
        // the tensor-core variants' operator table (FP32 residual on affine meshes)
        bool has_tc = false;
        for (int v = 0; v < nv; ++v) has_tc = has_tc || (vs[v].flags & dgk::kTC);
        if (has_tc && c->d_fflux && c->precision == DG_PREC_MIXED_FP32 && !c->pm.general) {
            std::vector<uint16_t> op;
            if (dgk::tc_operator(c->p, c->tab.B.data(), op) &&
                (cudaMalloc((void**)&c->d_tcop, op.size() * sizeof(uint16_t)) != cudaSuccess ||
                 cudaMemcpy(c->d_tcop, op.data(), op.size() * sizeof(uint16_t), cudaMemcpyHostToDevice) != cudaSuccess)) {
                cudaGetLastError();
                cudaFree(c->d_tcop);
                c->d_tcop = nullptr;
            }
        }
        // the default variant again, now that face-kernel variants may match
        for (int v = 0; v < nv; ++v)
            if (variant_matches(c, v)) {
                c->variant = v;
                break;
            }
    }
    std::vector<int2> hs(std::max(1, c->nslices)), hr(std::max(1, c->nslices));
    for (int i = 0; i < c->nslices; ++i) {
        hs[i] = make_int2(plan.send_elem[i], plan.send_face[i]);
        hr[i] = make_int2(plan.recv_elem[i], plan.recv_face[i]);
    }
    bool ok = cudaMemcpy(c->d_conn, conn.data(), conn.size() * sizeof(int2), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_frec, frec.data(), frec.size() * sizeof(dgk::FaceRec), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_geo_class, c->pm.geo_class.data(), c->ne_alloc * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_halo_send, hs.data(), hs.size() * sizeof(int2), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_halo_recv, hr.data(), hr.size() * sizeof(int2), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_X0, c->pm.X0.data(), c->pm.X0.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
              (c->pm.cmap.empty() || cudaMemcpy(c->d_cmap, c->pm.cmap.data(), c->pm.cmap.size(), cudaMemcpyHostToDevice) == cudaSuccess) &&
              (!c->pm.general ||
               (cudaMemcpy(c->d_gjd, c->pm.gjd.data(), c->pm.gjd.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
                cudaMemcpy(c->d_gnrm, gnrm.data(), gnrm.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
                cudaMemcpy(c->d_gimm, gimm.data(), gimm.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
                cudaMemcpy(c->d_gnodes, c->pm.gnodes.data(), c->pm.gnodes.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess)) &&
              cudaMemset(c->d_status, 0, sizeof(unsigned)) == cudaSuccess &&
              cudaMemset(c->d_U0, 0, nstate * sizeof(double)) == cudaSuccess &&
              cudaMemset(c->d_acc, 0, nstate * sizeof(double)) == cudaSuccess;
    if (!ok) {
        c->err = std::string("table upload failed: ") + cudaGetErrorString(cudaGetLastError());
        return bail(DG_ERR_CUDA);
    }
    c->class_dtf.assign(ncls, 1.0);
    c->class_eref.assign(ncls, 0.0);
    if ((rc = upload_geometry(c, c->stream)) != DG_OK) return bail(rc);
    if (c->pm.general && c->precision == DG_PREC_MIXED_FP32 && (rc = unit_pressure_residual(c)) != DG_OK) return bail(rc);
    *out = c;
    return DG_OK;
}

void dgi::destroy_ctx(dg_ctx* c)
{
    if (!c) return;
    release(c);
    delete c;
}

// ===========================================================================
namespace {
// data values each initial condition / exact solution family reads (DG_IC_*)
constexpr int kIcData[] = {5, 0, 0, 9, 1};

}  // namespace

extern "C" {

int dg_create(const dg_case_desc* cd, const dg_mesh_desc* md, dg_ctx** out)
{
    return create_ctx(cd, md, nullptr, nullptr, out);
}

int dg_create_partitioned(const dg_case_desc* cd, const dg_mesh_desc* md, const dg_part_desc* part, dg_ctx** out)
{
    if (!part) return fail(nullptr, DG_ERR_ARG, "dg_create_partitioned: null partition");
    return create_ctx(cd, md, nullptr, part, out);
}

int dg_partition_periodic_box(const int n[3], const double x0[3], const double len[3], unsigned rotate_seed, int nparts,
                              int part, int axis, int* nnode, double* node_coords, int* nelem, unsigned* elem_to_node_ids,
                              int* nface, unsigned* interior_faces, int* nowned, int* ninterior, int* ghost_rank,
                              int* ghost_elem, int* global_elem)
{
    if (!n || !x0 || !len || !nnode || !nelem || !nface || !nowned || !ninterior) return DG_ERR_ARG;
    if (n[0] < 1 || n[1] < 1 || n[2] < 1 || 1LL * n[0] * n[1] * n[2] > (1LL << 30)) return DG_ERR_ARG;
    if (axis < 0 || axis > 2 || nparts < 1 || nparts > n[axis] || part < 0 || part >= nparts) return DG_ERR_ARG;
    try {
        const dgh::BoxMesh g = dgh::make_periodic_box(n, x0, len, rotate_seed);
        const dgh::LocalMesh lm = dgh::partition_mesh(g, dgh::slab_partition(n, nparts, axis), part);
        *nnode = lm.mesh.nnode;
        *nelem = lm.mesh.nelem;
        *nface = lm.mesh.nface;
        *nowned = lm.nowned;
        *ninterior = lm.ninterior;
        const bool none = !node_coords && !elem_to_node_ids && !interior_faces && !ghost_rank && !ghost_elem && !global_elem;
        if (none) return DG_OK;
        if (!node_coords || !elem_to_node_ids || !interior_faces || !ghost_rank || !ghost_elem || !global_elem)
            return DG_ERR_ARG;
        std::memcpy(node_coords, lm.mesh.coords.data(), lm.mesh.coords.size() * sizeof(double));
        std::memcpy(elem_to_node_ids, lm.mesh.e2n.data(), lm.mesh.e2n.size() * sizeof(unsigned));
        std::memcpy(interior_faces, lm.mesh.faces.data(), lm.mesh.faces.size() * sizeof(unsigned));
        std::copy(lm.ghost_rank.begin(), lm.ghost_rank.end(), ghost_rank);
        std::copy(lm.ghost_elem.begin(), lm.ghost_elem.end(), ghost_elem);
        std::copy(lm.global_elem.begin(), lm.global_elem.end(), global_elem);
    } catch (const std::exception&) {
        return DG_ERR_ARG;
    }
    return DG_OK;
}

int dg_halo_plan(const dg_mesh_desc* md, const dg_part_desc* part, int* npeers, int* peer_rank, int* peer_offset,
                 int* peer_count, int* nslices, int* send_elem, int* send_face, int* recv_elem, int* recv_face)
{
    g_create_error.clear();
    if (!md || !part || !npeers || !nslices) return fail(nullptr, DG_ERR_ARG, "dg_halo_plan: null argument");
    const int ng = md->nelem - part->nowned;
    if (part->nowned < 1 || ng < 0 || (ng > 0 && (!part->ghost_rank || !part->ghost_elem)) || !md->interior_faces)
        return fail(nullptr, DG_ERR_ARG, "dg_halo_plan: partition description out of range");
    std::vector<int> er(md->nelem, md->rank);
    for (int g = 0; g < ng; ++g) er[part->nowned + g] = part->ghost_rank[g];
    dgh::MeshView mv;
    mv.nnode = md->nnode;
    mv.nelem = md->nelem;
    mv.nface = md->nface;
    mv.rank = md->rank;
    mv.coords = md->node_coords;
    mv.e2n = md->elem_to_node_ids;
    mv.faces = md->interior_faces;
    mv.nowned = part->nowned;
    mv.elem_rank = er.data();
    dgh::HaloPlan plan;
    const std::string err = dgh::make_halo_plan(mv, part->ghost_elem, plan);
    if (!err.empty()) return fail(nullptr, DG_ERR_ARG, err);
    *npeers = static_cast<int>(plan.peer_rank.size());
    *nslices = static_cast<int>(plan.send_elem.size());
    if (peer_rank) std::copy(plan.peer_rank.begin(), plan.peer_rank.end(), peer_rank);
    if (peer_offset) std::copy(plan.peer_offset.begin(), plan.peer_offset.end(), peer_offset);
    if (peer_count) std::copy(plan.peer_count.begin(), plan.peer_count.end(), peer_count);
    if (send_elem) std::copy(plan.send_elem.begin(), plan.send_elem.end(), send_elem);
    if (send_face) std::copy(plan.send_face.begin(), plan.send_face.end(), send_face);
    if (recv_elem) std::copy(plan.recv_elem.begin(), plan.recv_elem.end(), recv_elem);
    if (recv_face) std::copy(plan.recv_face.begin(), plan.recv_face.end(), recv_face);
    return DG_OK;
}

int dg_halo_num_peers(const dg_ctx* c) { return c ? static_cast<int>(c->peer_rank.size()) : 0; }

int dg_halo_peer(const dg_ctx* c, int i, int* rank, int* offset, int* count)
{
    if (!c || i < 0 || i >= static_cast<int>(c->peer_rank.size())) return DG_ERR_ARG;
    if (rank) *rank = c->peer_rank[i];
    if (offset) *offset = c->peer_offset[i];
    if (count) *count = c->peer_count[i];
    return DG_OK;
}

int dg_halo_slice_doubles(const dg_ctx* c) { return c ? 5 * (c->p + 1) * (c->p + 1) : 0; }

namespace {

double* rk_buffer(dg_ctx* c, int buf)
{
    return buf == DG_BUF_U0 ? c->d_U0 : buf == DG_BUF_STAGE_A ? c->d_Ua : buf == DG_BUF_STAGE_B ? c->d_Ub : nullptr;
}

int halo_launch(dg_ctx* c, int buf, double* d_data, void* stream, bool pack)
{
    double* U = rk_buffer(c, buf);
    if (!U) return fail(c, DG_ERR_ARG, "unknown state buffer");
    if (c->nslices == 0) return DG_OK;
    if (!d_data) return fail(c, DG_ERR_ARG, "null halo buffer");
    DG_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    const long long total = 5LL * (c->p + 1) * (c->p + 1) * c->nslices;
    const int grid = static_cast<int>(std::min<long long>((total + 255) / 256, 4096));
    if (pack) halo_pack_kernel<<<grid, 256, 0, s>>>(U, c->d_halo_send, c->nslices, c->p + 1, d_data);
    else halo_unpack_kernel<<<grid, 256, 0, s>>>(U, c->d_halo_recv, c->nslices, c->p + 1, d_data);
    DG_CUDA(c, cudaGetLastError());
    return DG_OK;
}

}  // namespace

int dg_halo_pack(dg_ctx* c, int buf, double* d_send, void* stream)
{
    dgi::NvtxRange nvtx_("dg_halo_pack");
    if (!c) return DG_ERR_ARG;
    return halo_launch(c, buf, d_send, stream, true);
}

int dg_halo_unpack(dg_ctx* c, int buf, const double* d_recv, void* stream)
{
    dgi::NvtxRange nvtx_("dg_halo_unpack");
    if (!c) return DG_ERR_ARG;
    return halo_launch(c, buf, const_cast<double*>(d_recv), stream, false);
}

int dg_rk4_stage(dg_ctx* c, int stage, double dt, int range)
{
    dgi::NvtxRange nvtx_("dg_rk4_stage");
    if (!c || stage < 1 || stage > 4 || range < 0 || range > 2 || !std::isfinite(dt))
        return fail(c, DG_ERR_ARG, "dg_rk4_stage: bad argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    const int e0 = range == 2 ? c->ninterior : 0, e1 = range == 1 ? c->ninterior : c->ne;
    switch (stage) {
        case 1: return launch_stage(c, dgk::kModeRK1, c->d_U0, c->d_U0, c->d_Ua, dt, e0, e1);
        case 2: return launch_stage(c, dgk::kModeRK2, c->d_Ua, c->d_U0, c->d_Ub, dt, e0, e1);
        case 3: return launch_stage(c, dgk::kModeRK3, c->d_Ub, c->d_U0, c->d_Ua, dt, e0, e1);
        default: return launch_stage(c, dgk::kModeRK4, c->d_Ua, c->d_U0, c->d_U0, dt, e0, e1);
    }
}

void* dg_stream(dg_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

void dg_destroy(dg_ctx* ctx) { destroy_ctx(ctx); }

const char* dg_last_error(const dg_ctx* ctx)
{
    if (!ctx) return g_create_error.c_str();
    return ctx->err.c_str();
}

int dg_num_basis(const dg_ctx* ctx) { return ctx ? ctx->nb : 0; }
int dg_num_elements(const dg_ctx* ctx) { return ctx ? ctx->ne : 0; }

namespace {

// the FP32 residual's energy reference follows the uploaded state
int set_energy_reference(dg_ctx* c, const double* Uc)
{
    if (c->precision != DG_PREC_MIXED_FP32) return DG_OK;
    const double e = energy_reference(c, Uc, c->ne);
    if (c->class_eref.empty() || c->class_eref[0] == e) return DG_OK;
    std::fill(c->class_eref.begin(), c->class_eref.end(), e);
    return upload_geometry(c, c->stream);
}

}  // namespace

int dg_set_state(dg_ctx* c, const double* Uc)
{
    dgi::NvtxRange nvtx_("dg_set_state");
    if (!c || !Uc) return fail(c, DG_ERR_ARG, "dg_set_state: null argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    const int rc = set_energy_reference(c, Uc);
    if (rc) return rc;
    return upload_state_host_layout(c, Uc, c->d_U0);
}

int dg_get_state(dg_ctx* c, double* Uc)
{
    dgi::NvtxRange nvtx_("dg_get_state");
    if (!c || !Uc) return fail(c, DG_ERR_ARG, "dg_get_state: null argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    return download_host_layout(c, c->d_U0, Uc);
}

int dg_residual(dg_ctx* c, double* res)
{
    dgi::NvtxRange nvtx_("dg_residual");
    if (!c || !res) return fail(c, DG_ERR_ARG, "dg_residual: null argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    int rc = launch_stage(c, dgk::kModeResidual, c->d_U0, c->d_U0, c->d_acc, 0.0);
    if (rc) return rc;
    rc = download_host_layout(c, c->d_acc, res);
    if (rc) return rc;
    return check_status(c);
}

int dg_mass_inverse_residual(dg_ctx* c, double dt, double* dU)
{
    dgi::NvtxRange nvtx_("dg_mass_inverse_residual");
    if (!c || !dU || !std::isfinite(dt)) return fail(c, DG_ERR_ARG, "dg_mass_inverse_residual: bad argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    int rc = launch_stage(c, dgk::kModeMassInv, c->d_U0, c->d_U0, c->d_acc, dt);
    if (rc) return rc;
    rc = download_host_layout(c, c->d_acc, dU);
    if (rc) return rc;
    return check_status(c);
}

namespace {

// one RK stage as c->chunks element chunks (contexts without ghosts, a
// face-kernel variant): the face launches of the chunks on the second stream
// (they read only the stage input), each chunk's stage launch on the main
// stream after its face launch, so a chunk's face kernel runs beside the
// previous chunk's stage kernel and its fluxes are read soon after they are
// written.  `stage` (0..3) picks the stage's events.
int launch_stage_chunked(dg_ctx* c, int stage, int mode, const double* Us, const double* U0, double* out, double dt)
{
    const dgk::StageVariant* vs = nullptr;
    dgk::stage_variants(c->p, &vs);
    const dgk::StageVariant& sv = vs[c->variant];
    const int C = c->chunks;
    if (!sv.face_launch || C <= 1 || c->face_key.size() != static_cast<size_t>(c->nface) ||
        c->chunk_ev.size() < static_cast<size_t>(4 * (C + 1)))
        return launch_stage(c, mode, Us, U0, out, dt);
    cudaEvent_t* ev = c->chunk_ev.data() + stage * (C + 1);
    StageArgs a;
    stage_args(c, mode, Us, U0, out, dt, 0, c->ne, a);
    DG_CUDA(c, cudaEventRecord(ev[0], c->stream));
    DG_CUDA(c, cudaStreamWaitEvent(c->stream2, ev[0], 0));
    std::vector<int> e_at(C + 1);
    for (int k = 0; k <= C; ++k) e_at[k] = static_cast<int>(static_cast<long long>(c->ne) * k / C);
    const int fb = sv.face_batch;
    for (int k = 0; k < C; ++k) {
        const int f0 = static_cast<int>(std::lower_bound(c->face_key.begin(), c->face_key.end(), e_at[k]) - c->face_key.begin());
        const int f1 = static_cast<int>(std::lower_bound(c->face_key.begin(), c->face_key.end(), e_at[k + 1]) - c->face_key.begin());
        a.face_begin = f0;
        a.nface = f1;
        if (f1 > f0) DG_CUDA(c, sv.face_launch(a, std::min(c->variant_face_grid[c->variant], (f1 - f0 + fb - 1) / fb), c->stream2));
        DG_CUDA(c, cudaEventRecord(ev[k + 1], c->stream2));
    }
    for (int k = 0; k < C; ++k) {
        DG_CUDA(c, cudaStreamWaitEvent(c->stream, ev[k + 1], 0));
        a.e_begin = e_at[k];
        a.ne = e_at[k + 1];
        const int batches = (e_at[k + 1] - e_at[k] + sv.E - 1) / sv.E;
        if (batches > 0) DG_CUDA(c, sv.launch(a, std::min(c->variant_grid[c->variant], batches), c->stream));
    }
    return DG_OK;
}

int prepare_rk4_graph(dg_ctx* c, double dt)
{
    if (c->graph_exec && c->graph_dt == dt) return DG_OK;
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    // kernel attributes and the grid are set outside the capture
    int rc = prepare_variant(c, c->variant);
    if (rc) return rc;
    DG_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    if (c->chunks > 1) {
        rc = launch_stage_chunked(c, 0, dgk::kModeRK1, c->d_U0, c->d_U0, c->d_Ua, dt);
        if (!rc) rc = launch_stage_chunked(c, 1, dgk::kModeRK2, c->d_Ua, c->d_U0, c->d_Ub, dt);
        if (!rc) rc = launch_stage_chunked(c, 2, dgk::kModeRK3, c->d_Ub, c->d_U0, c->d_Ua, dt);
        if (!rc) rc = launch_stage_chunked(c, 3, dgk::kModeRK4, c->d_Ua, c->d_U0, c->d_U0, dt);
    } else {
        rc = launch_stage(c, dgk::kModeRK1, c->d_U0, c->d_U0, c->d_Ua, dt);
        if (!rc) rc = launch_stage(c, dgk::kModeRK2, c->d_Ua, c->d_U0, c->d_Ub, dt);
        if (!rc) rc = launch_stage(c, dgk::kModeRK3, c->d_Ub, c->d_U0, c->d_Ua, dt);
        if (!rc) rc = launch_stage(c, dgk::kModeRK4, c->d_Ua, c->d_U0, c->d_U0, dt);
    }
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (ce != cudaSuccess) return fail(c, DG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    c->graph = g;
    DG_CUDA(c, cudaGraphInstantiate(&c->graph_exec, c->graph, 0));
    c->graph_dt = dt;
    return DG_OK;
}

}  // namespace

int dg_rk4_steps_timed(dg_ctx* c, double dt, int nsteps, double* device_ms)
{
    dgi::NvtxRange nvtx_("dg_rk4_steps_timed");
    if (!c || nsteps < 0 || !device_ms || !std::isfinite(dt)) return fail(c, DG_ERR_ARG, "dg_rk4_steps_timed: bad argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    int rc = prepare_rk4_graph(c, dt);
    if (rc) return rc;
    cudaEvent_t ev[2];
    DG_CUDA(c, cudaEventCreate(&ev[0]));
    if (cudaEventCreate(&ev[1]) != cudaSuccess) { cudaEventDestroy(ev[0]); return fail(c, DG_ERR_CUDA, "cudaEventCreate"); }
    cudaError_t ce = cudaEventRecord(ev[0], c->stream);
    for (int s = 0; s < nsteps && ce == cudaSuccess; ++s) ce = cudaGraphLaunch(c->graph_exec, c->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[1], c->stream);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[1]);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, ev[0], ev[1]);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (ce != cudaSuccess) return fail(c, DG_ERR_CUDA, std::string("timed RK4: ") + cudaGetErrorString(ce));
    *device_ms = ms;
    return check_status(c);
}

int dg_num_stage_variants(int order)
{
    const dgk::StageVariant* vs = nullptr;
    return dgk::stage_variants(order, &vs);
}

int dg_stage_variant_info(int order, int v, int* elems_per_cta, int* threads_per_cta, int* groups, int* precision)
{
    const dgk::StageVariant* vs = nullptr;
    const int nv = dgk::stage_variants(order, &vs);
    if (v < 0 || v >= nv) return DG_ERR_ARG;
    if (elems_per_cta) *elems_per_cta = vs[v].E;
    if (threads_per_cta) *threads_per_cta = vs[v].NT;
    if (groups) *groups = vs[v].G;
    if (precision) *precision = vs[v].fp32 ? DG_PREC_MIXED_FP32 : DG_PREC_FP64;
    return DG_OK;
}

int dg_stage_variant_flags(int order, int v, int* flags)
{
    const dgk::StageVariant* vs = nullptr;
    const int nv = dgk::stage_variants(order, &vs);
    if (v < 0 || v >= nv || !flags) return DG_ERR_ARG;
    *flags = vs[v].flags;
    return DG_OK;
}

int dg_set_stage_variant(dg_ctx* c, int v)
{
    if (!c) return DG_ERR_ARG;
    if (v < 0 || v >= dg_num_stage_variants(c->p)) return fail(c, DG_ERR_ARG, "stage variant index out of range");
    if (!variant_matches(c, v))
        return fail(c, DG_ERR_ARG, "stage variant has the other residual precision or geometry kind");
    if (v != c->variant) {
        c->variant = v;
        if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
        if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    }
    return DG_OK;
}

int dg_get_stage_variant(const dg_ctx* c) { return c ? c->variant : -1; }

int dg_set_stage_chunks(dg_ctx* c, int chunks)
{
    if (!c || chunks < 1 || chunks > 64) return fail(c, DG_ERR_ARG, "dg_set_stage_chunks: chunks must be 1..64");
    if (chunks > 1 && (c->face_key.size() != static_cast<size_t>(c->nface) || !c->d_fflux))
        return fail(c, DG_ERR_UNSUPPORTED, "dg_set_stage_chunks: contexts with ghosts or without a face list");
    DG_CUDA(c, cudaSetDevice(c->device));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (chunks > 1 && !c->stream2) DG_CUDA(c, cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking));
    while (c->chunk_ev.size() < static_cast<size_t>(4 * (chunks + 1))) {
        cudaEvent_t e;
        DG_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->chunk_ev.push_back(e);
    }
    if (c->chunks != chunks) {
        c->chunks = chunks;
        // the RK4 graph holds the launch sequence
        if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
        if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    }
    return DG_OK;
}

int dg_get_stage_chunks(const dg_ctx* c) { return c ? c->chunks : -1; }

int dg_tune_stage(dg_ctx* c, int reps, int* best, double* ms_per_variant)
{
    dgi::NvtxRange nvtx_("dg_tune_stage");
    if (!c || reps < 1) return fail(c, DG_ERR_ARG, "dg_tune_stage: bad argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    const int nv = dg_num_stage_variants(c->p);
    const int keep = c->variant;
    int winner = keep;
    double best_ms = 1e300;
    cudaEvent_t ev[2];
    DG_CUDA(c, cudaEventCreate(&ev[0]));
    if (cudaEventCreate(&ev[1]) != cudaSuccess) { cudaEventDestroy(ev[0]); return fail(c, DG_ERR_CUDA, "cudaEventCreate"); }
    int rc = DG_OK;
    for (int v = 0; v < nv && rc == DG_OK; ++v) {
        if (!variant_matches(c, v)) {
            if (ms_per_variant) ms_per_variant[v] = -1.0;
            continue;
        }
        c->variant = v;
        // one untimed launch, then `reps` timed ones of an RK2 stage (reads the
        // stage state, U0 and the accumulator, writes the accumulator and an
        // output): the traffic of a real stage.  The output goes to scratch and
        // the accumulator is dead between steps, so the state is unchanged.
        rc = launch_stage(c, dgk::kModeRK2, c->d_U0, c->d_U0, c->d_out, 1e-3);
        if (rc) break;
        cudaEventRecord(ev[0], c->stream);
        for (int r = 0; r < reps && rc == DG_OK; ++r) rc = launch_stage(c, dgk::kModeRK2, c->d_U0, c->d_U0, c->d_out, 1e-3);
        cudaEventRecord(ev[1], c->stream);
        if (cudaEventSynchronize(ev[1]) != cudaSuccess) { rc = fail(c, DG_ERR_CUDA, "tuning launch failed"); break; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        const double per = ms / reps;
        if (ms_per_variant) ms_per_variant[v] = per;
        if (per < best_ms) { best_ms = per; winner = v; }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    c->variant = keep;
    if (rc) return rc;
    rc = dg_set_stage_variant(c, winner);
    if (rc) return rc;
    if (best) *best = winner;
    return DG_OK;
}

int dg_rk4_steps(dg_ctx* c, double dt, int nsteps)
{
    dgi::NvtxRange nvtx_("dg_rk4_steps");
    if (!c || nsteps < 0 || !std::isfinite(dt)) return fail(c, DG_ERR_ARG, "dg_rk4_steps: bad argument");
    if (nsteps == 0) return DG_OK;
    DG_CUDA(c, cudaSetDevice(c->device));
    int rc = prepare_rk4_graph(c, dt);
    if (rc) return rc;
    for (int s = 0; s < nsteps; ++s) DG_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_status(c);
}

int dg_fe_steps(dg_ctx* c, double dt, int nsteps)
{
    dgi::NvtxRange nvtx_("dg_fe_steps");
    if (!c || nsteps < 0 || !std::isfinite(dt)) return fail(c, DG_ERR_ARG, "dg_fe_steps: bad argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    for (int s = 0; s < nsteps; ++s) {
        int rc = launch_stage(c, dgk::kModeFE, c->d_U0, c->d_U0, c->d_Ua, dt);
        if (rc) return rc;
        std::swap(c->d_U0, c->d_Ua);
    }
    // the RK4 graph captured the old buffer addresses
    if (nsteps > 0 && c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        cudaGraphDestroy(c->graph);
        c->graph_exec = nullptr;
        c->graph = nullptr;
    }
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_status(c);
}

int dg_project_ic(dg_ctx* c, int ic_type, const double* data, int ndata, double t, double* Uc)
{
    dgi::NvtxRange nvtx_("dg_project_ic");
    if (!c) return fail(c, DG_ERR_ARG, "dg_project_ic: null context");
    if (ic_type < DG_IC_UNIFORM || ic_type > DG_IC_TAYLOR_GREEN) return fail(c, DG_ERR_ARG, "unknown initial condition");
    if (ndata < kIcData[ic_type] || (ndata > 0 && !data))
        return fail(c, DG_ERR_ARG, "initial condition needs more data values");
    double d[16] = {0};
    for (int i = 0; i < ndata && i < 16; ++i) d[i] = data[i];
    DG_CUDA(c, cudaSetDevice(c->device));
    int rc = project_ic_device(c, ic_type, d, 16, t, c->gamma, c->R, 0, c->ne);
    if (rc) return rc;
    const bool mixed = c->precision == DG_PREC_MIXED_FP32;
    if (!Uc && !mixed) {
        DG_CUDA(c, cudaStreamSynchronize(c->stream));
        return DG_OK;
    }
    // a host copy for the caller, and for the mixed residual's energy reference
    std::vector<double> tmp;
    double* host = Uc;
    if (!host) {
        tmp.resize(static_cast<size_t>(c->ne) * c->nb * 5);
        host = tmp.data();
    }
    rc = download_range(c, c->d_U0, host, 0, c->ne);
    if (rc) return rc;
    return set_energy_reference(c, host);
}

int dg_l2_error(dg_ctx* c, int ic_type, const double* data, int ndata, double t, double* err)
{
    dgi::NvtxRange nvtx_("dg_l2_error");
    if (!c || !err) return fail(c, DG_ERR_ARG, "dg_l2_error: null argument");
    if (ic_type < DG_IC_UNIFORM || ic_type > DG_IC_TAYLOR_GREEN) return fail(c, DG_ERR_ARG, "unknown exact solution");
    if (ndata < kIcData[ic_type] || (ndata > 0 && !data))
        return fail(c, DG_ERR_ARG, "exact solution needs more data values");
    DG_CUDA(c, cudaSetDevice(c->device));
    double sums[5];
    int rc = run_reduce(c, 0, ic_type, data, ndata, t, sums, 0, c->ne, c->gamma, c->R);
    if (rc) return rc;
    for (int v = 0; v < 5; ++v) err[v] = std::sqrt(sums[v] / c->pm.volume);
    return DG_OK;
}

int dg_kinetic_energy(dg_ctx* c, double* ke)
{
    dgi::NvtxRange nvtx_("dg_kinetic_energy");
    if (!c || !ke) return fail(c, DG_ERR_ARG, "dg_kinetic_energy: null argument");
    DG_CUDA(c, cudaSetDevice(c->device));
    double sums[5];
    int rc = run_reduce(c, 1, 0, nullptr, 0, 0.0, sums, 0, c->ne, c->gamma, c->R);
    if (rc) return rc;
    *ke = sums[0] / c->pm.volume;
    return DG_OK;
}

namespace {

// The bounded mbarrier wait of the tensor-core kernel (tc::mbar_wait) on a
// barrier that nothing completes, or that thread 0 completes first: the wait
// gives up after `limit` SM cycles and the kernel reports kStatusTimeout and
// returns. No asynchronous copy is attached to the barrier, so a wait that
// gives up leaves nothing in flight.
__global__ void bounded_wait_probe_kernel(long long limit, int arrive, unsigned* status, long long* cycles)
{
    __shared__ alignas(8) unsigned long long bar;
    const uint32_t b = dgk::tc::smem_u32(&bar);
    if (threadIdx.x == 0) {
        dgk::tc::mbar_init(b, 1);
        dgk::tc::mbar_fence_init();
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0) dgk::tc::mbar_arrive(b);
    const long long t0 = clock64();
    const bool ok = __syncthreads_and(dgk::tc::mbar_wait(b, 0, limit));
    if (threadIdx.x == 0) {
        cycles[0] = clock64() - t0;
        status[0] = ok ? 0u : dgk::kStatusTimeout;
        dgk::tc::mbar_inval(b);
    }
}

}  // namespace

int dg_probe_bounded_wait(int device, long long limit_cycles, int arrive, long long* waited_cycles)
{
    g_create_error.clear();
    if (limit_cycles < 0 || limit_cycles > 4000000000LL)
        return fail(nullptr, DG_ERR_ARG, "dg_probe_bounded_wait: limit must be 0 .. 4e9 SM cycles (about 2 s)");
    int prev = 0;
    cudaError_t ce = cudaGetDevice(&prev);
    if (ce == cudaSuccess) ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return fail(nullptr, DG_ERR_CUDA, std::string("dg_probe_bounded_wait: ") + cudaGetErrorString(ce));
    void* buf = nullptr;
    unsigned st = 0;
    long long cyc = 0;
    ce = cudaMalloc(&buf, 16);
    if (ce == cudaSuccess) {
        long long* d_cycles = static_cast<long long*>(buf);
        unsigned* d_status = reinterpret_cast<unsigned*>(d_cycles + 1);
        bounded_wait_probe_kernel<<<1, 32>>>(limit_cycles, arrive ? 1 : 0, d_status, d_cycles);
        ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = cudaMemcpy(&st, d_status, sizeof(st), cudaMemcpyDeviceToHost);
        if (ce == cudaSuccess) ce = cudaMemcpy(&cyc, d_cycles, sizeof(cyc), cudaMemcpyDeviceToHost);
        const cudaError_t fe = cudaFree(buf);
        if (ce == cudaSuccess) ce = fe;
    }
    (void)cudaSetDevice(prev);
    if (ce != cudaSuccess) return fail(nullptr, DG_ERR_CUDA, std::string("dg_probe_bounded_wait: ") + cudaGetErrorString(ce));
    if (waited_cycles) *waited_cycles = cyc;
    if (st & dgk::kStatusTimeout)
        return fail(nullptr, DG_ERR_TIMEOUT,
                    "dg_probe_bounded_wait: the bounded wait gave up after " + std::to_string(cyc) + " SM cycles");
    return DG_OK;
}

int dg_kinetic_energy_noalloc(int order, int nelem, const double* d_state, const double* d_djac, double* d_ke,
                              void* stream)
{
    g_create_error.clear();
    if (order < 0 || order > dgk::kMaxP) return fail(nullptr, DG_ERR_ARG, "dg_kinetic_energy_noalloc: order must be 0..5");
    if (nelem <= 0 || !d_state || !d_djac || !d_ke)
        return fail(nullptr, DG_ERR_ARG, "dg_kinetic_energy_noalloc: null pointer or empty mesh");
    if (nelem > kNoAllocMaxElems)
        return fail(nullptr, DG_ERR_ARG,
                    "dg_kinetic_energy_noalloc: " + std::to_string(nelem) + " elements exceed the allocation-free limit of " +
                        std::to_string(kNoAllocMaxElems) + " (16384 blocks of 64 elements in a 256 KB static scratch array)");
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return fail(nullptr, DG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    if (dev < 0 || dev >= 64) return fail(nullptr, DG_ERR_UNSUPPORTED, "device ordinal above 63");
    // every buffer must be memory of the current device: a pointer of another
    // device (or a host pointer) would fault asynchronously, after DG_OK
    const void* bufs[3] = {d_state, d_djac, d_ke};
    const char* names[3] = {"d_state", "d_djac", "d_ke"};
    for (int i = 0; i < 3; ++i) {
        cudaPointerAttributes at{};
        ce = cudaPointerGetAttributes(&at, bufs[i]);
        if (ce != cudaSuccess) {
            (void)cudaGetLastError();
            return fail(nullptr, DG_ERR_ARG, std::string("dg_kinetic_energy_noalloc: ") + names[i] +
                                                  " is not a CUDA pointer: " + cudaGetErrorString(ce));
        }
        if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
            return fail(nullptr, DG_ERR_ARG, std::string("dg_kinetic_energy_noalloc: ") + names[i] + " is not device memory");
        if (at.device != dev)
            return fail(nullptr, DG_ERR_ARG, std::string("dg_kinetic_energy_noalloc: ") + names[i] + " is memory of device " +
                                                  std::to_string(at.device) + ", not of the current device " +
                                                  std::to_string(dev));
    }
    double* scratch = nullptr;
    {
        // one-time set-up per device, with that device current: basis tables
        // and the device address of the static scratch array
        std::lock_guard<std::mutex> lk(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            dg_ctx tmp;
            tmp.device = dev;
            if (load_constant_tables(&tmp) != DG_OK) return fail(nullptr, DG_ERR_CUDA, tmp.err);
            void* p = nullptr;
            ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (ce != cudaSuccess || !p)
                return fail(nullptr, DG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
            g_noalloc_ptr[dev] = static_cast<double*>(p);
        }
        scratch = g_noalloc_ptr[dev];
    }
    const int nblocks = (nelem + kNoAllocElemsPerBlock - 1) / kNoAllocElemsPerBlock;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (order) {
        case 0: ke_partials_noalloc<0><<<nblocks, 256, 0, s>>>(d_state, d_djac, nelem, scratch); break;
        case 1: ke_partials_noalloc<1><<<nblocks, 256, 0, s>>>(d_state, d_djac, nelem, scratch); break;
        case 2: ke_partials_noalloc<2><<<nblocks, 256, 0, s>>>(d_state, d_djac, nelem, scratch); break;
        case 3: ke_partials_noalloc<3><<<nblocks, 256, 0, s>>>(d_state, d_djac, nelem, scratch); break;
        case 4: ke_partials_noalloc<4><<<nblocks, 256, 0, s>>>(d_state, d_djac, nelem, scratch); break;
        default: ke_partials_noalloc<5><<<nblocks, 256, 0, s>>>(d_state, d_djac, nelem, scratch); break;
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(nullptr, DG_ERR_CUDA, std::string("kinetic-energy partials: ") + cudaGetErrorString(ce));
    ke_finalize_noalloc<<<1, 256, 0, s>>>(scratch, nblocks, d_ke);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(nullptr, DG_ERR_CUDA, std::string("kinetic-energy finalise: ") + cudaGetErrorString(ce));
    return DG_OK;
}

int dg_total_volume(const dg_ctx* c, double* vol)
{
    if (!c || !vol) return DG_ERR_ARG;
    *vol = c->pm.volume;
    return DG_OK;
}

int dg_status(dg_ctx* c, unsigned* flags)
{
    if (!c || !flags) return fail(c, DG_ERR_ARG, "dg_status: null argument");
    unsigned st = 0;
    DG_CUDA(c, cudaSetDevice(c->device));
    DG_CUDA(c, cudaMemcpy(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    DG_CUDA(c, cudaMemset(c->d_status, 0, sizeof(unsigned)));
    *flags = st | c->status_accum;
    c->status_accum = 0;
    return DG_OK;
}

int dg_sync(dg_ctx* c)
{
    if (!c) return DG_ERR_ARG;
    DG_CUDA(c, cudaSetDevice(c->device));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

void* dg_device_state(dg_ctx* c) { return c ? c->d_U0 : nullptr; }

int dg_mesh_periodic_box(const int n[3], const double x0[3], const double len[3], unsigned rotate_seed,
                         int* nnode, double* node_coords, int* nelem, unsigned* elem_to_node_ids, int* nface,
                         unsigned* interior_faces)
{
    if (!n || !x0 || !len || !nnode || !nelem || !nface) return DG_ERR_ARG;
    if (n[0] < 1 || n[1] < 1 || n[2] < 1) return DG_ERR_ARG;
    const long long ne = 1LL * n[0] * n[1] * n[2];
    if (ne > (1LL << 30)) return DG_ERR_ARG;
    *nnode = (n[0] + 1) * (n[1] + 1) * (n[2] + 1);
    *nelem = static_cast<int>(ne);
    *nface = static_cast<int>(3 * ne);
    if (!node_coords && !elem_to_node_ids && !interior_faces) return DG_OK;
    if (!node_coords || !elem_to_node_ids || !interior_faces) return DG_ERR_ARG;
    try {
        dgh::BoxMesh b = dgh::make_periodic_box(n, x0, len, rotate_seed);
        std::memcpy(node_coords, b.coords.data(), b.coords.size() * sizeof(double));
        std::memcpy(elem_to_node_ids, b.e2n.data(), b.e2n.size() * sizeof(unsigned));
        std::memcpy(interior_faces, b.faces.data(), b.faces.size() * sizeof(unsigned));
    } catch (const std::exception&) {
        return DG_ERR_ARG;
    }
    return DG_OK;
}

int dg_gauss_legendre(int n, double* x, double* w)
{
    if (n < 1 || n > 64 || !x || !w) return DG_ERR_ARG;
    std::vector<double> xv, wv;
    dgh::gauss_legendre(n, xv, wv);
    std::copy(xv.begin(), xv.end(), x);
    std::copy(wv.begin(), wv.end(), w);
    return DG_OK;
}

int dg_face_orientation_order(int orient, int npts, int* order)
{
    if (orient < 0 || orient > 7 || npts < 1 || !order) return DG_ERR_ARG;
    std::vector<int> o;
    dgh::face_orientation_order(orient, npts, o);
    std::copy(o.begin(), o.end(), order);
    return DG_OK;
}

int dg_basis_tables(int p, double* B, double* D, double* Minv)
{
    if (p < 0 || p > 8) return DG_ERR_ARG;
    const dgh::Tables1D t = dgh::make_tables(p);
    if (B) std::copy(t.B.begin(), t.B.end(), B);
    if (D) std::copy(t.D.begin(), t.D.end(), D);
    if (Minv) std::copy(t.Minv.begin(), t.Minv.end(), Minv);
    return DG_OK;
}

int dg_cfl_time_step(dg_ctx* c, const double* Uc, double cfl, double* dt)
{
    dgi::NvtxRange nvtx_("dg_cfl_time_step");
    if (!c || !Uc || !dt || !(cfl > 0.0)) return fail(c, DG_ERR_ARG, "dg_cfl_time_step: bad argument");
    const double v = dgh::cfl_time_step(c->pm, c->p, c->gamma, Uc, cfl, 0, c->ne);
    if (!(v > 0.0)) return fail(c, DG_ERR_NONPHYSICAL, "state has non-positive density or pressure");
    *dt = v;
    return DG_OK;
}

}  // extern "C"
