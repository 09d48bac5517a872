// dg_2d.cu -- the 2D quadrilateral path (Solver<2> with LagrangeQuad): the
// residual and RK stage on periodic meshes of parallelograms, FP64, one warp
// per element, and its C ABI (dg2d_* in dg_b200.h).
//
// Reference path replaced (the 2D instantiation of the 3D path's functions,
// citations relative to the reference root): Solver<2>::get_residual
// (src/solver/base.cpp:401-561) with evaluate_state (helpers.cpp:185-198),
// VolumeFluxesFunctor (flux_functors_impl.h:46-115), the grad-basis^T
// contraction (solver/tools.cpp:7-35), construct_face_states / the face flux
// functor / construct_flux_state (base.cpp:287-374,
// flux_functors_impl.h:168-264), the face lift (tools.cpp:38-63),
// mult_inv_mass_matrix (tools.cpp:124-139) and the RK4 / FE stage updates
// (stepper.cpp:23-142).
//
// Per element (one warp; shared memory per warp, no block barriers):
//   load U [4][nb];  x and y interpolation to the (p+2)^2 Gauss points
//   (sum-factorised: B is the 1D basis at the volume points); the Euler flux
//   at each point (dgp::interior_flux on the state with a zero third
//   momentum: the reference's 2D flux, functions.cpp:43-61, is the 3D one
//   without the third components), times (ijac djac)(x) w_q; the x and y
//   contractions with the 1D derivative and basis into the residual; for each
//   of the 4 edges and each of its p+1 Gauss points the element's trace and
//   the neighbour's (only the edge's p+1 nodes carry the trace of an
//   equidistant Lagrange basis, the others vanish there exactly, so the sums
//   equal the reference's dense B_f U term by term), the numerical flux in the
//   reference's L/R roles with the left element's normal (dgp::flux_*, the
//   2D Lax-Friedrichs / HLLC of functions.cpp:196-297 being the 3D ones on
//   (nx, ny, 0)), times the edge weight, -F on the left and +F on the right;
//   the lift of the four edges into the residual; the Kronecker inverse mass
//   over det J and the fused RK / FE update.  Each edge flux is evaluated by
//   both of its elements in the same argument order, so both see the same
//   value.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dg_b200.h"
#include "../host/numerics.h"
#include "dg_physics.cuh"

namespace dgi {
int fail(dg_ctx* c, int code, const std::string& msg);
}

namespace d2 {

constexpr int kNS = 4;
constexpr int kMaxN = 6, kMaxM = 7;
constexpr int kWarps = 4;  // elements in flight per CTA

enum Mode : int { kResidual = 0, kRK1 = 2, kRK2 = 3, kRK3 = 4, kRK4 = 5, kFE = 6 };
enum Status : unsigned { kRho = 1u, kPressure = 2u, kNaN = 4u, kHLLC = 8u };

// the order's tables (copied to shared memory by every CTA)
struct Tab {
    double B[kMaxM * kMaxN], D[kMaxM * kMaxN], wv[kMaxM];  // volume: [q][i]
    double FB[4 * kMaxN * kMaxN];                          // [f][j][m]: edge node m at edge point j
    double fw[kMaxN];                                      // edge weights
    double Minv[kMaxN * kMaxN];                            // 1D inverse mass
    int fnode[4 * kMaxN];                                  // [f][m]: basis index of edge node m (ascending)
    int lift[4 * kMaxN * kMaxN];                           // [f][b]: m with fnode[f][m] == b, else -1
};

struct Geo {
    double jd[4];  // (ijac * djac)[d1][d2]
    double idj;    // 1 / djac
    double pad[3];
};

struct Face {
    int nbr;
    int code;  // neighbour face | role << 2 (0 left, 1 right) | flip << 3 | my orientation << 4
    double N[2];
};

struct Args {
    const double* Us;
    double* out;
    const double* U0;
    double* acc;
    const Geo* geo;
    const Face* faces;
    const Tab* tab;
    unsigned* status;
    int ne, mode, flux;
    double dt, gamma;
};

template <int P>
struct Cfg {
    static constexpr int N = P + 1, M = P + 2, NB = N * N, NQ = M * M, NF = P + 1;
    // per-warp shared memory (doubles): U, R, the interpolation / contraction
    // area (T1 + Uq, later H), the point fluxes G, the edge fluxes Fe
    static constexpr int kU = 0, kR = kU + kNS * NB, kA = kR + kNS * NB;
    static constexpr int kAsz = kNS * N * M + kNS * M * M;  // >= 2 kNS M N (M > N)
    static constexpr int kG = kA + kAsz, kFe = kG + 2 * kNS * NQ, kEnd = kFe + 4 * NF * kNS;
};

constexpr size_t kTabDoubles = (sizeof(Tab) + 7) / 8;

template <int P>
__global__ void __launch_bounds__(32 * kWarps) stage2d_kernel(const Args a)
{
    using C = Cfg<P>;
    constexpr int N = C::N, M = C::M, NB = C::NB, NQ = C::NQ, NF = C::NF;
    extern __shared__ double sm[];
    Tab& T = *reinterpret_cast<Tab*>(sm);
    {
        const double* src = reinterpret_cast<const double*>(a.tab);
        for (int i = threadIdx.x; i < static_cast<int>(kTabDoubles); i += blockDim.x) sm[i] = src[i];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* W = sm + kTabDoubles + static_cast<size_t>(warp) * C::kEnd;
    double* U = W + C::kU;
    double* R = W + C::kR;
    double* T1 = W + C::kA;               // [v][j][qx]
    double* Uq = T1 + kNS * N * M;        // [v][qy][qx]
    double* H = W + C::kA;                // [d][v][qy][i], after Uq is dead
    double* G = W + C::kG;                // [d][v][qy][qx]
    double* Fe = W + C::kFe;              // [f][j][v]
    unsigned status = 0;
    const double gam = a.gamma;
    for (int e = blockIdx.x * kWarps + warp; e < a.ne; e += gridDim.x * kWarps) {
        const double* Ue = a.Us + static_cast<size_t>(e) * kNS * NB;
        for (int i = lane; i < kNS * NB; i += 32) U[i] = Ue[i];
        const Geo g = a.geo[e];
        __syncwarp();
        // x interpolation: T1[v][j][qx] = sum_i B[qx][i] U[v][j][i]
        for (int t = lane; t < kNS * N * M; t += 32) {
            const int qx = t % M, j = (t / M) % N, v = t / (M * N);
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < N; ++i) s += T.B[qx * N + i] * U[v * NB + j * N + i];
            T1[t] = s;
        }
        __syncwarp();
        // y interpolation: Uq[v][qy][qx] = sum_j B[qy][j] T1[v][j][qx]
        for (int t = lane; t < kNS * NQ; t += 32) {
            const int qx = t % M, qy = (t / M) % M, v = t / NQ;
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < N; ++j) s += T.B[qy * N + j] * T1[(v * N + j) * M + qx];
            Uq[t] = s;
        }
        __syncwarp();
        // pointwise flux times (ijac djac)(x) w
        for (int q = lane; q < NQ; q += 32) {
            const double u5[5] = {Uq[q], Uq[NQ + q], Uq[2 * NQ + q], 0.0, Uq[3 * NQ + q]};
            double F[15];
            dgp::interior_flux(gam, u5, F);
            const double p = dgp::pressure(gam, u5);
            if (!(u5[0] > 0.0)) status |= kRho;
            if (!(p > 0.0)) status |= kPressure;
            if (u5[0] != u5[0] || p != p) status |= kNaN;
            const double w = T.wv[q % M] * T.wv[q / M];
            constexpr int s3[4] = {0, 1, 2, 4};
#pragma unroll
            for (int v = 0; v < kNS; ++v) {
                const double fx = F[s3[v]], fy = F[5 + s3[v]];
#pragma unroll
                for (int d = 0; d < 2; ++d) G[(d * kNS + v) * NQ + q] = (fx * g.jd[d * 2 + 0] + fy * g.jd[d * 2 + 1]) * w;
            }
        }
        __syncwarp();
        // x contraction: H0 = D^T along x of G0, H1 = B^T along x of G1
        for (int t = lane; t < 2 * kNS * M * N; t += 32) {
            const int i = t % N, qy = (t / N) % M, dv = t / (N * M);
            const double* Op = dv < kNS ? T.D : T.B;
            const double* g0 = G + dv * NQ + qy * M;
            double s = 0.0;
#pragma unroll
            for (int qx = 0; qx < M; ++qx) s += Op[qx * N + i] * g0[qx];
            H[t] = s;
        }
        __syncwarp();
        // y contraction into the residual
        for (int t = lane; t < kNS * NB; t += 32) {
            const int i = t % N, j = (t / N) % N, v = t / NB;
            const double* h0 = H + (v * M) * N + i;
            const double* h1 = H + ((kNS + v) * M) * N + i;
            double s = 0.0;
#pragma unroll
            for (int qy = 0; qy < M; ++qy) s += T.B[qy * N + j] * h0[qy * N] + T.D[qy * N + j] * h1[qy * N];
            R[t] = s;
        }
        // edges: one lane per (face, point)
        if (lane < 4 * NF) {
            const int f = lane / NF, j = lane % NF;
            const Face fr = a.faces[static_cast<size_t>(e) * 4 + f];
            if (fr.nbr < 0) {
#pragma unroll
                for (int v = 0; v < kNS; ++v) Fe[(f * NF + j) * kNS + v] = 0.0;
            } else {
                const int nf = fr.code & 3, role = (fr.code >> 2) & 1, flip = (fr.code >> 3) & 1, mine = (fr.code >> 4) & 1;
                const int jn = flip ? NF - 1 - j : j;
                const int q = mine ? NF - 1 - j : j;  // the face's quadrature point
                const double* Un = a.Us + static_cast<size_t>(fr.nbr) * kNS * NB;
                double uo[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, un[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                constexpr int s3[4] = {0, 1, 2, 4};
    #pragma unroll
                for (int v = 0; v < kNS; ++v) {
                    double so = 0.0, sn = 0.0;
    #pragma unroll
                    for (int m = 0; m < N; ++m) {
                        so += T.FB[(f * N + j) * N + m] * U[v * NB + T.fnode[f * N + m]];
                        sn += T.FB[(nf * N + jn) * N + m] * __ldg(Un + v * NB + T.fnode[nf * N + m]);
                    }
                    uo[s3[v]] = so;
                    un[s3[v]] = sn;
                }
                const double* UL = role == 0 ? uo : un;
                const double* UR = role == 0 ? un : uo;
                const double N3[3] = {fr.N[0], fr.N[1], 0.0};
                double F5[5];
                if (a.flux == DG_FLUX_HLLC) {
                    if (!dgp::flux_hllc(gam, UL, UR, N3, F5)) status |= kHLLC;
                } else {
                    dgp::flux_lax_friedrichs(gam, UL, UR, N3, F5);
                }
                const double sgn = role == 0 ? -1.0 : 1.0;
    #pragma unroll
                for (int v = 0; v < kNS; ++v) Fe[(f * NF + j) * kNS + v] = sgn * (F5[s3[v]] * T.fw[q]);
            }
        }
        __syncwarp();
        // lift of the four edges: the edge nodes of b, face by face
        for (int t = lane; t < kNS * NB; t += 32) {
            const int b = t % NB, v = t / NB;
            double s = 0.0;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const int m = T.lift[f * kMaxN * kMaxN + b];
                if (m >= 0)
#pragma unroll
                    for (int j = 0; j < NF; ++j) s += T.FB[(f * N + j) * N + m] * Fe[(f * NF + j) * kNS + v];
            }
            R[t] += s;
        }
        __syncwarp();
        double* Oe = a.out + static_cast<size_t>(e) * kNS * NB;
        if (a.mode == kResidual) {
            for (int i = lane; i < kNS * NB; i += 32) Oe[i] = R[i];
            __syncwarp();
            continue;
        }
        // inverse mass: (Minv x Minv) R / det J, x then y; then the stage update
        for (int t = lane; t < kNS * NB; t += 32) {
            const int i = t % N, jv = t / N;
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += T.Minv[i * N + k] * R[jv * N + k];
            T1[t] = s;
        }
        __syncwarp();
        const double* U0e = a.U0 + static_cast<size_t>(e) * kNS * NB;
        double* Ae = a.acc + static_cast<size_t>(e) * kNS * NB;
        for (int t = lane; t < kNS * NB; t += 32) {
            const int i = t % N, j = (t / N) % N, v = t / NB;
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += T.Minv[j * N + k] * T1[(v * N + k) * N + i];
            const double kk = a.dt * (s * g.idj);
            const double u0 = U0e[t];
            switch (a.mode) {
                case kRK1: Ae[t] = kk; Oe[t] = 0.5 * kk + u0; break;
                case kRK2: Ae[t] = Ae[t] + 2.0 * kk; Oe[t] = 0.5 * kk + u0; break;
                case kRK3: Ae[t] = Ae[t] + 2.0 * kk; Oe[t] = 1.0 * kk + u0; break;
                case kRK4: Oe[t] = u0 + (1.0 / 6.0) * (Ae[t] + kk); break;
                default: Oe[t] = u0 + kk; break;
            }
        }
        __syncwarp();
    }
    // one atomic per warp
    for (int off = 16; off > 0; off >>= 1) status |= __shfl_xor_sync(0xffffffffu, status, off);
    if (lane == 0 && status) atomicOr(a.status, status);
}

template <int P>
size_t smem_bytes()
{
    return (kTabDoubles + static_cast<size_t>(kWarps) * Cfg<P>::kEnd) * sizeof(double);
}

using KernelFn = void (*)(const Args);
KernelFn kernel_of(int p)
{
    switch (p) {
        case 0: return stage2d_kernel<0>;
        case 1: return stage2d_kernel<1>;
        case 2: return stage2d_kernel<2>;
        case 3: return stage2d_kernel<3>;
        case 4: return stage2d_kernel<4>;
        default: return stage2d_kernel<5>;
    }
}
size_t smem_of(int p)
{
    switch (p) {
        case 0: return smem_bytes<0>();
        case 1: return smem_bytes<1>();
        case 2: return smem_bytes<2>();
        case 3: return smem_bytes<3>();
        case 4: return smem_bytes<4>();
        default: return smem_bytes<5>();
    }
}

// ---------------- host ----------------

// corner nodes of an edge in traversal order (get_points_on_face_quadrilateral,
// shape.cpp:69-122)
constexpr int kFaceNodes[4][2] = {{0, 1}, {1, 3}, {3, 2}, {2, 0}};
constexpr double kRefX[4] = {-1., 1., -1., 1.}, kRefY[4] = {-1., -1., 1., 1.};

// the order's tables: volume rule of (p+2) points per direction, edge rule of
// p+1 points, edge traces from the 2D basis at the edge points computed as
// get_points_on_face_quadrilateral and get_lagrange_basis_val_2D do
bool make_tab(int p, const dgh::Tables1D& t1, Tab& T)
{
    std::memset(&T, 0, sizeof(T));
    const int n = p + 1, m = p + 2, nf = p + 1;
    for (int q = 0; q < m; ++q) {
        T.wv[q] = t1.wq[q];
        for (int i = 0; i < n; ++i) {
            T.B[q * n + i] = t1.B[q * n + i];
            T.D[q * n + i] = t1.D[q * n + i];
        }
    }
    for (int i = 0; i < n * n; ++i) T.Minv[i] = t1.Minv[i];
    std::vector<double> s, w;
    dgh::gauss_legendre(nf, s, w);
    for (int q = 0; q < nf; ++q) T.fw[q] = w[q];
    const std::vector<double> xn = dgh::equidistant_nodes(n);
    for (int i = 0; i < 4 * kMaxN * kMaxN; ++i) T.lift[i] = -1;
    for (int f = 0; f < 4; ++f) {
        const int a = kFaceNodes[f][0], b = kFaceNodes[f][1];
        std::vector<double> val(static_cast<size_t>(nf) * n * n);
        for (int q = 0; q < nf; ++q) {
            const double b1 = (s[q] + 1.) / 2., b0 = 1.0 - b1;
            const double x = b0 * kRefX[a] + b1 * kRefX[b], y = b0 * kRefY[a] + b1 * kRefY[b];
            double vx[kMaxN], vy[kMaxN], gx[kMaxN], gy[kMaxN];
            dgh::lagrange_1d(x, xn, vx, gx);
            dgh::lagrange_1d(y, xn, vy, gy);
            for (int jj = 0; jj < n; ++jj)
                for (int ii = 0; ii < n; ++ii) val[(static_cast<size_t>(q) * n + jj) * n + ii] = vx[ii] * vy[jj];
        }
        // the edge's nodes (basis index j n + i with j = 0, i = p, j = p, i = 0
        // on faces 0..3), in ascending index; every other basis function
        // vanishes on the edge (its Lagrange factor in the normal direction is
        // zero at the edge's coordinate)
        int cnt = 0;
        for (int k = 0; k < n * n; ++k) {
            const int i = k % n, jj = k / n;
            const bool on = (f == 0 && jj == 0) || (f == 1 && i == p) || (f == 2 && jj == p) || (f == 3 && i == 0);
            if (!on) {
                for (int q = 0; q < nf; ++q)
                    if (std::fabs(val[static_cast<size_t>(q) * n * n + k]) > 1e-14) return false;
                continue;
            }
            T.fnode[f * n + cnt] = k;
            T.lift[f * kMaxN * kMaxN + k] = cnt;
            for (int q = 0; q < nf; ++q) T.FB[(f * n + q) * n + cnt] = val[static_cast<size_t>(q) * n * n + k];
            ++cnt;
        }
        if (cnt != n) return false;
    }
    return true;
}

}  // namespace d2

struct dg_ctx2d {
    int device = 0, p = 0, nb = 1, ne = 0, nnode = 0, flux = 0;
    double gamma = 1.4, R = 1.0;
    cudaStream_t stream = nullptr;
    double *d_U0 = nullptr, *d_Ua = nullptr, *d_Ub = nullptr, *d_acc = nullptr, *d_res = nullptr;
    d2::Geo* d_geo = nullptr;
    d2::Face* d_faces = nullptr;
    d2::Tab* d_tab = nullptr;
    unsigned* d_status = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double graph_dt = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int grid = 1;
    size_t smem = 0;
    dgh::Tables1D t1;
    std::vector<double> coords;  // [nnode][2]
    std::vector<unsigned> e2n;   // [ne][4]
    std::vector<double> djac;    // [ne]
    std::string err;
};

namespace {

int fail2(dg_ctx2d* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    else dgi::fail(nullptr, code, msg);
    return code;
}

#define DG2_CUDA(c, call)                                                                               \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail2((c), DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void release(dg_ctx2d* c)
{
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    cudaFree(c->d_U0);
    cudaFree(c->d_Ua);
    cudaFree(c->d_Ub);
    cudaFree(c->d_acc);
    cudaFree(c->d_res);
    cudaFree(c->d_geo);
    cudaFree(c->d_faces);
    cudaFree(c->d_tab);
    cudaFree(c->d_status);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
}

int launch(dg_ctx2d* c, const double* Us, double* out, int mode, double dt)
{
    d2::Args a{};
    a.Us = Us;
    a.out = out;
    a.U0 = c->d_U0;
    a.acc = c->d_acc;
    a.geo = c->d_geo;
    a.faces = c->d_faces;
    a.tab = c->d_tab;
    a.status = c->d_status;
    a.ne = c->ne;
    a.mode = mode;
    a.flux = c->flux;
    a.dt = dt;
    a.gamma = c->gamma;
    d2::kernel_of(c->p)<<<c->grid, 32 * d2::kWarps, c->smem, c->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DG_OK : fail2(c, DG_ERR_CUDA, std::string("stage2d launch: ") + cudaGetErrorString(e));
}

int check_status(dg_ctx2d* c)
{
    unsigned s = 0;
    DG2_CUDA(c, cudaMemcpyAsync(&s, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    DG2_CUDA(c, cudaStreamSynchronize(c->stream));
    if (s) return fail2(c, DG_ERR_NONPHYSICAL, "non-physical state (status " + std::to_string(s) + ")");
    return DG_OK;
}

// host layout [ne][nb][4] <-> device layout [ne][4][nb]
void to_device_layout(const double* h, double* d, int ne, int nb)
{
    for (int e = 0; e < ne; ++e)
        for (int b = 0; b < nb; ++b)
            for (int v = 0; v < d2::kNS; ++v)
                d[(static_cast<size_t>(e) * d2::kNS + v) * nb + b] = h[(static_cast<size_t>(e) * nb + b) * d2::kNS + v];
}
void to_host_layout(const double* d, double* h, int ne, int nb)
{
    for (int e = 0; e < ne; ++e)
        for (int b = 0; b < nb; ++b)
            for (int v = 0; v < d2::kNS; ++v)
                h[(static_cast<size_t>(e) * nb + b) * d2::kNS + v] = d[(static_cast<size_t>(e) * d2::kNS + v) * nb + b];
}

// the IC families of the 2D path at (x, y): the 3D families at (x, y, 0)
// without their third momentum; DG_IC_VORTEX_2D is the x-y family centred at
// the origin with no period (the reference's 2D vortex, functions.cpp:94-145)
bool ic_state(int type, const double* data, int ndata, double gamma, double R, double x, double y, double t, double* U4)
{
    double x3[3] = {x, y, 0.0}, U5[5], d[9] = {0, 0, 0, 0, 0, 0, 0, 1e300, 1e300};
    if (type == DG_IC_VORTEX_2D) {
        for (int i = 0; i < 5 && i < ndata; ++i) d[i] = data[i];
        dgp::initial_state(DG_IC_VORTEX_XY, d, gamma, R, x3, t, U5);
    } else if (type == DG_IC_UNIFORM) {
        const double u[5] = {data[0], data[1], data[2], 0.0, data[3]};
        dgp::initial_state(DG_IC_UNIFORM, u, gamma, R, x3, t, U5);
    } else if (type == DG_IC_VORTEX_XY) {
        dgp::initial_state(DG_IC_VORTEX_XY, data, gamma, R, x3, t, U5);
    } else {
        return false;
    }
    U4[0] = U5[0];
    U4[1] = U5[1];
    U4[2] = U5[2];
    U4[3] = U5[4];
    return true;
}

bool ic_args_ok(int type, int ndata)
{
    if (type == DG_IC_VORTEX_2D) return ndata >= 5;
    if (type == DG_IC_UNIFORM) return ndata >= 4;
    if (type == DG_IC_VORTEX_XY) return ndata >= 9;
    return false;
}

// (x, y) of reference point (xi, eta) of element e (the bilinear map,
// MeshTools::ref_to_phys, mesh/tools.cpp:19-26)
void ref_to_phys(const dg_ctx2d* c, int e, double xi, double eta, double& x, double& y)
{
    const double gv[4] = {0.25 * (1 - xi) * (1 - eta), 0.25 * (1 + xi) * (1 - eta), 0.25 * (1 - xi) * (1 + eta),
                          0.25 * (1 + xi) * (1 + eta)};
    x = y = 0.0;
    for (int n = 0; n < 4; ++n) {
        x += gv[n] * c->coords[2 * c->e2n[4 * e + n]];
        y += gv[n] * c->coords[2 * c->e2n[4 * e + n] + 1];
    }
}

int prepare_graph(dg_ctx2d* c, double dt)
{
    if (c->graph_exec && c->graph_dt == dt) return DG_OK;
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    DG2_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = launch(c, c->d_U0, c->d_Ua, d2::kRK1, dt);
    if (!rc) rc = launch(c, c->d_Ua, c->d_Ub, d2::kRK2, dt);
    if (!rc) rc = launch(c, c->d_Ub, c->d_Ua, d2::kRK3, dt);
    if (!rc) rc = launch(c, c->d_Ua, c->d_U0, d2::kRK4, dt);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (ce != cudaSuccess) return fail2(c, DG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    c->graph = g;
    DG2_CUDA(c, cudaGraphInstantiate(&c->graph_exec, c->graph, 0));
    c->graph_dt = dt;
    return DG_OK;
}

}  // namespace

extern "C" {

int dg2d_create(const dg_case_desc* cd, const dg_mesh2d_desc* md, dg_ctx2d** out)
{
    if (!cd || !md || !out) return fail2(nullptr, DG_ERR_ARG, "dg2d_create: null argument");
    *out = nullptr;
    if (cd->order < 0 || cd->order > 5) return fail2(nullptr, DG_ERR_UNSUPPORTED, "dg2d_create: order must be 0..5");
    if (cd->flux != DG_FLUX_LAX_FRIEDRICHS && cd->flux != DG_FLUX_HLLC) return fail2(nullptr, DG_ERR_ARG, "dg2d_create: unknown flux");
    if (cd->precision != DG_PREC_FP64) return fail2(nullptr, DG_ERR_UNSUPPORTED, "dg2d_create: the 2D path is FP64");
    if (!(cd->gamma > 1.0)) return fail2(nullptr, DG_ERR_ARG, "dg2d_create: gamma must exceed 1");
    if (md->nnode < 4 || md->nelem < 1 || md->nface < 0 || !md->node_coords || !md->elem_to_node_ids ||
        (md->nface > 0 && !md->interior_faces))
        return fail2(nullptr, DG_ERR_ARG, "dg2d_create: empty mesh");
    if (2LL * md->nface > 4LL * md->nelem) return fail2(nullptr, DG_ERR_ARG, "dg2d_create: more faces than element edges");
    dg_ctx2d* c = new dg_ctx2d();
    c->device = cd->device;
    c->p = cd->order;
    c->nb = (c->p + 1) * (c->p + 1);
    c->ne = md->nelem;
    c->nnode = md->nnode;
    c->flux = cd->flux;
    c->gamma = cd->gamma;
    c->R = cd->gas_constant;
    auto bail = [&](int code, const std::string& msg) {
        dgi::fail(nullptr, code, "dg2d_create: " + msg);
        release(c);
        delete c;
        return code;
    };
    try {
        c->coords.assign(md->node_coords, md->node_coords + 2 * static_cast<size_t>(md->nnode));
        c->e2n.assign(md->elem_to_node_ids, md->elem_to_node_ids + 4 * static_cast<size_t>(md->nelem));
        for (unsigned v : c->e2n)
            if (v >= static_cast<unsigned>(md->nnode)) return bail(DG_ERR_ARG, "node id out of range");
        // geometry: parallelograms only (constant Jacobian), as the reference
        // computes it per point (basis/tools.cpp:42-66, linear_algebra.cpp:99-107)
        std::vector<d2::Geo> geo(c->ne);
        c->djac.resize(c->ne);
        for (int e = 0; e < c->ne; ++e) {
            double X[4][2];
            for (int n = 0; n < 4; ++n)
                for (int d = 0; d < 2; ++d) X[n][d] = c->coords[2 * c->e2n[4 * e + n] + d];
            double scale = 0.0;
            for (int n = 0; n < 4; ++n) scale = std::max(scale, std::max(std::fabs(X[n][0] - X[0][0]), std::fabs(X[n][1] - X[0][1])));
            // parallelograms up to the rounding of mesh files' coordinates
            // (1e-9 of the element's size); the Jacobian of the bilinear map
            // at the element's centre, the mean of its Jacobian over the element
            for (int d = 0; d < 2; ++d)
                if (std::fabs((X[3][d] - X[2][d]) - (X[1][d] - X[0][d])) > 1e-9 * scale)
                    return bail(DG_ERR_UNSUPPORTED, "element " + std::to_string(e) + " is not a parallelogram");
            double jac[4];
            for (int i = 0; i < 2; ++i) {
                jac[i * 2 + 0] = 0.25 * ((X[1][i] - X[0][i]) + (X[3][i] - X[2][i]));
                jac[i * 2 + 1] = 0.25 * ((X[2][i] - X[0][i]) + (X[3][i] - X[1][i]));
            }
            const double det = jac[0] * jac[3] - jac[1] * jac[2];
            if (!(det > 0.0)) return bail(DG_ERR_ARG, "element " + std::to_string(e) + " has a non-positive Jacobian");
            const double ij[4] = {jac[3] / det, -jac[1] / det, -jac[2] / det, jac[0] / det};
            for (int k = 0; k < 4; ++k) geo[e].jd[k] = ij[k] * det;
            geo[e].idj = 1.0 / det;
            c->djac[e] = det;
        }
        // faces: per element and local face, the neighbour, its face, the
        // roles and orientations, and the left element's normal; an edge that
        // is no interior face (a boundary edge of a non-periodic mesh) keeps
        // nbr = -1 and adds nothing, as the reference's residual, which loops
        // over the interior faces only (base.cpp:470-561)
        std::vector<d2::Face> faces(4 * static_cast<size_t>(c->ne), d2::Face{-1, 0, {0.0, 0.0}});
        std::vector<char> seen(4 * static_cast<size_t>(c->ne), 0);
        for (int f = 0; f < md->nface; ++f) {
            const unsigned* r = md->interior_faces + 8 * static_cast<size_t>(f);
            if (r[0] != static_cast<unsigned>(md->rank) || r[4] != static_cast<unsigned>(md->rank))
                return bail(DG_ERR_ARG, "face rows must carry this rank");
            const unsigned eL = r[1], fL = r[2], oL = r[3], eR = r[5], fR = r[6], oR = r[7];
            if (eL >= static_cast<unsigned>(c->ne) || eR >= static_cast<unsigned>(c->ne) || fL > 3 || fR > 3 || oL > 1 || oR > 1)
                return bail(DG_ERR_ARG, "face row " + std::to_string(f) + " out of range");
            if (seen[4 * eL + fL] || seen[4 * eR + fR] || (eL == eR && fL == fR))
                return bail(DG_ERR_ARG, "an element face appears twice");
            seen[4 * eL + fL] = seen[4 * eR + fR] = 1;
            // normal (dy/ds, -dx/ds) of the left element's edge with the
            // LagrangeSeg p = 1 gradient (-1/2, 1/2) (shape.cpp:154-210)
            const int a = d2::kFaceNodes[fL][0], b = d2::kFaceNodes[fL][1];
            const double* XA = &c->coords[2 * c->e2n[4 * eL + a]];
            const double* XB = &c->coords[2 * c->e2n[4 * eL + b]];
            const double g0 = -0.5, g1 = 0.5;
            const double dx = XA[0] * g0 + XB[0] * g1, dy = XA[1] * g0 + XB[1] * g1;
            const double N0 = 1.0 * dy, N1 = -1.0 * 1.0 * dx;
            const int flip = static_cast<int>(oL ^ oR);
            faces[4 * eL + fL] = d2::Face{static_cast<int>(eR), static_cast<int>(fR) | (0 << 2) | (flip << 3) | (static_cast<int>(oL) << 4), {N0, N1}};
            faces[4 * eR + fR] = d2::Face{static_cast<int>(eL), static_cast<int>(fL) | (1 << 2) | (flip << 3) | (static_cast<int>(oR) << 4), {N0, N1}};
        }
        c->t1 = dgh::make_tables(c->p);
        d2::Tab tab;
        if (!d2::make_tab(c->p, c->t1, tab)) return bail(DG_ERR_ARG, "edge trace tables");

        if (cudaSetDevice(c->device) != cudaSuccess) return bail(DG_ERR_CUDA, "cudaSetDevice failed");
        const size_t nstate = static_cast<size_t>(c->ne) * d2::kNS * c->nb * sizeof(double);
        bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreate(&c->ev0) == cudaSuccess && cudaEventCreate(&c->ev1) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_U0, nstate) == cudaSuccess && cudaMalloc((void**)&c->d_Ua, nstate) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_Ub, nstate) == cudaSuccess && cudaMalloc((void**)&c->d_acc, nstate) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_res, nstate) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_geo, geo.size() * sizeof(d2::Geo)) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_faces, faces.size() * sizeof(d2::Face)) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_tab, sizeof(d2::Tab)) == cudaSuccess &&
                  cudaMalloc((void**)&c->d_status, sizeof(unsigned)) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            return bail(DG_ERR_NOMEM, "device allocation failed");
        }
        ok = cudaMemcpy(c->d_geo, geo.data(), geo.size() * sizeof(d2::Geo), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(c->d_faces, faces.data(), faces.size() * sizeof(d2::Face), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(c->d_tab, &tab, sizeof(d2::Tab), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemset(c->d_status, 0, sizeof(unsigned)) == cudaSuccess &&
             cudaMemset(c->d_U0, 0, nstate) == cudaSuccess && cudaMemset(c->d_acc, 0, nstate) == cudaSuccess;
        if (!ok) return bail(DG_ERR_CUDA, "device upload failed");
        c->smem = d2::smem_of(c->p);
        if (cudaFuncSetAttribute(reinterpret_cast<const void*>(d2::kernel_of(c->p)), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(c->smem)) != cudaSuccess)
            return bail(DG_ERR_CUDA, "kernel attribute");
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(d2::kernel_of(c->p)),
                                                      32 * d2::kWarps, c->smem);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        const int need = (c->ne + d2::kWarps - 1) / d2::kWarps;
        c->grid = std::max(1, std::min(need, std::max(1, per_sm) * std::max(1, sms)));
    } catch (const std::bad_alloc&) {
        return bail(DG_ERR_NOMEM, "host allocation failed");
    }
    *out = c;
    return DG_OK;
}

void dg2d_destroy(dg_ctx2d* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    release(c);
    delete c;
}

const char* dg2d_last_error(const dg_ctx2d* c) { return c ? c->err.c_str() : dg_last_error(nullptr); }

int dg2d_num_basis(const dg_ctx2d* c) { return c ? c->nb : 0; }

int dg2d_set_state(dg_ctx2d* c, const double* Uc)
{
    if (!c || !Uc) return fail2(c, DG_ERR_ARG, "dg2d_set_state: null argument");
    std::vector<double> d(static_cast<size_t>(c->ne) * d2::kNS * c->nb);
    to_device_layout(Uc, d.data(), c->ne, c->nb);
    DG2_CUDA(c, cudaSetDevice(c->device));
    DG2_CUDA(c, cudaMemcpyAsync(c->d_U0, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    DG2_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int dg2d_get_state(dg_ctx2d* c, double* Uc)
{
    if (!c || !Uc) return fail2(c, DG_ERR_ARG, "dg2d_get_state: null argument");
    std::vector<double> d(static_cast<size_t>(c->ne) * d2::kNS * c->nb);
    DG2_CUDA(c, cudaSetDevice(c->device));
    DG2_CUDA(c, cudaMemcpyAsync(d.data(), c->d_U0, d.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DG2_CUDA(c, cudaStreamSynchronize(c->stream));
    to_host_layout(d.data(), Uc, c->ne, c->nb);
    return DG_OK;
}

int dg2d_residual(dg_ctx2d* c, double* res)
{
    if (!c || !res) return fail2(c, DG_ERR_ARG, "dg2d_residual: null argument");
    DG2_CUDA(c, cudaSetDevice(c->device));
    int rc = launch(c, c->d_U0, c->d_res, d2::kResidual, 0.0);
    if (rc) return rc;
    std::vector<double> d(static_cast<size_t>(c->ne) * d2::kNS * c->nb);
    DG2_CUDA(c, cudaMemcpyAsync(d.data(), c->d_res, d.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((rc = check_status(c))) return rc;
    to_host_layout(d.data(), res, c->ne, c->nb);
    return DG_OK;
}

int dg2d_rk4_steps_timed(dg_ctx2d* c, double dt, int nsteps, double* device_ms)
{
    if (!c || nsteps < 0 || !(dt > 0.0)) return fail2(c, DG_ERR_ARG, "dg2d_rk4_steps: bad argument");
    DG2_CUDA(c, cudaSetDevice(c->device));
    int rc = prepare_graph(c, dt);
    if (rc) return rc;
    DG2_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (int s = 0; s < nsteps; ++s) DG2_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
    DG2_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    if ((rc = check_status(c))) return rc;
    if (device_ms) {
        float ms = 0.f;
        DG2_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        *device_ms = ms;
    }
    return DG_OK;
}

int dg2d_rk4_steps(dg_ctx2d* c, double dt, int nsteps) { return dg2d_rk4_steps_timed(c, dt, nsteps, nullptr); }

int dg2d_fe_steps(dg_ctx2d* c, double dt, int nsteps)
{
    if (!c || nsteps < 0 || !(dt > 0.0)) return fail2(c, DG_ERR_ARG, "dg2d_fe_steps: bad argument");
    DG2_CUDA(c, cudaSetDevice(c->device));
    // the update reads its neighbours' stage state, so it writes another buffer
    for (int s = 0; s < nsteps; ++s) {
        int rc = launch(c, c->d_U0, c->d_Ua, d2::kFE, dt);
        if (rc) return rc;
        std::swap(c->d_U0, c->d_Ua);
    }
    if (nsteps % 2 && c->graph_exec) {
        // the RK4 graph captured the old buffer addresses
        cudaGraphExecDestroy(c->graph_exec);
        cudaGraphDestroy(c->graph);
        c->graph_exec = nullptr;
        c->graph = nullptr;
    }
    return check_status(c);
}

int dg2d_project_ic(dg_ctx2d* c, int ic_type, const double* data, int ndata, double t, double* Uc)
{
    if (!c || (ndata > 0 && !data) || !ic_args_ok(ic_type, ndata)) return fail2(c, DG_ERR_ARG, "dg2d_project_ic: bad initial condition");
    // init_state_from_fcn + L2 projection (base.cpp:113-223) on the
    // (2 max(p,1) + 2)^2 rule, the Kronecker inverse mass over det J
    const dgh::Tables1D& tb = c->t1;
    const int n = c->p + 1, me = tb.me, nb = c->nb;
    std::vector<double> U(static_cast<size_t>(c->ne) * nb * d2::kNS);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < c->ne; ++e) {
        std::vector<double> f(static_cast<size_t>(me) * me * d2::kNS), rhs(static_cast<size_t>(nb) * d2::kNS), tmp(rhs.size());
        for (int qy = 0; qy < me; ++qy)
            for (int qx = 0; qx < me; ++qx) {
                double x, y, Ue[4];
                ref_to_phys(c, e, tb.xe[qx], tb.xe[qy], x, y);
                ic_state(ic_type, data, ndata, c->gamma, c->R, x, y, t, Ue);
                const double cw = (tb.we[qx] * tb.we[qy]) * c->djac[e];
                for (int v = 0; v < d2::kNS; ++v) f[(static_cast<size_t>(qy) * me + qx) * d2::kNS + v] = Ue[v] * cw;
            }
        for (int b = 0; b < nb; ++b)
            for (int v = 0; v < d2::kNS; ++v) {
                const int i = b % n, j = b / n;
                double acc = 0.0;
                for (int qy = 0; qy < me; ++qy)
                    for (int qx = 0; qx < me; ++qx)
                        acc += (tb.Be[qx * n + i] * tb.Be[qy * n + j]) * f[(static_cast<size_t>(qy) * me + qx) * d2::kNS + v];
                rhs[b * d2::kNS + v] = acc;
            }
        for (int b = 0; b < nb; ++b)
            for (int v = 0; v < d2::kNS; ++v) {
                const int i = b % n, j = b / n;
                double acc = 0.0;
                for (int k = 0; k < n; ++k) acc += tb.Minv[i * n + k] * rhs[(j * n + k) * d2::kNS + v];
                tmp[b * d2::kNS + v] = acc;
            }
        for (int b = 0; b < nb; ++b)
            for (int v = 0; v < d2::kNS; ++v) {
                const int i = b % n, j = b / n;
                double acc = 0.0;
                for (int k = 0; k < n; ++k) acc += tb.Minv[j * n + k] * tmp[(k * n + i) * d2::kNS + v];
                U[(static_cast<size_t>(e) * nb + b) * d2::kNS + v] = acc / c->djac[e];
            }
    }
    if (Uc) std::copy(U.begin(), U.end(), Uc);
    return dg2d_set_state(c, U.data());
}

int dg2d_l2_error(dg_ctx2d* c, int ic_type, const double* data, int ndata, double t, double* err)
{
    if (!c || !err || (ndata > 0 && !data) || !ic_args_ok(ic_type, ndata)) return fail2(c, DG_ERR_ARG, "dg2d_l2_error: bad argument");
    std::vector<double> U(static_cast<size_t>(c->ne) * c->nb * d2::kNS);
    int rc = dg2d_get_state(c, U.data());
    if (rc) return rc;
    // get_error (post/main.cpp:30-201) on the (2 max(p,1) + 2)^2 rule,
    // normalised by the volume of the volume rule (mesh/tools.cpp:28-36)
    const dgh::Tables1D& tb = c->t1;
    const int n = c->p + 1, me = tb.me, nb = c->nb;
    std::vector<double> per(static_cast<size_t>(c->ne) * d2::kNS, 0.0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < c->ne; ++e) {
        const double* Ue = U.data() + static_cast<size_t>(e) * nb * d2::kNS;
        double acc[4] = {0, 0, 0, 0};
        for (int qy = 0; qy < me; ++qy)
            for (int qx = 0; qx < me; ++qx) {
                double Uq[4] = {0, 0, 0, 0}, Ex[4], x, y;
                for (int b = 0; b < nb; ++b) {
                    const double bv = tb.Be[qx * n + b % n] * tb.Be[qy * n + b / n];
                    for (int v = 0; v < d2::kNS; ++v) Uq[v] += bv * Ue[b * d2::kNS + v];
                }
                ref_to_phys(c, e, tb.xe[qx], tb.xe[qy], x, y);
                ic_state(ic_type, data, ndata, c->gamma, c->R, x, y, t, Ex);
                const double w = (tb.we[qx] * tb.we[qy]) * c->djac[e];
                for (int v = 0; v < d2::kNS; ++v) acc[v] += (Uq[v] - Ex[v]) * (Uq[v] - Ex[v]) * w;
            }
        for (int v = 0; v < d2::kNS; ++v) per[static_cast<size_t>(e) * d2::kNS + v] = acc[v];
    }
    double tot[4] = {0, 0, 0, 0}, vol = 0.0, wsum = 0.0;
    for (int q = 0; q < c->p + 2; ++q)
        for (int r = 0; r < c->p + 2; ++r) wsum += tb.wq[r] * tb.wq[q];
    for (int e = 0; e < c->ne; ++e) {
        for (int v = 0; v < d2::kNS; ++v) tot[v] += per[static_cast<size_t>(e) * d2::kNS + v];
        vol += wsum * c->djac[e];
    }
    for (int v = 0; v < d2::kNS; ++v) err[v] = std::sqrt(tot[v] / vol);
    return DG_OK;
}

int dg2d_status(dg_ctx2d* c, unsigned* flags)
{
    if (!c || !flags) return fail2(c, DG_ERR_ARG, "dg2d_status: null argument");
    DG2_CUDA(c, cudaSetDevice(c->device));
    DG2_CUDA(c, cudaMemcpyAsync(flags, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    DG2_CUDA(c, cudaStreamSynchronize(c->stream));
    return *flags ? DG_ERR_NONPHYSICAL : DG_OK;
}

}  // extern "C"
