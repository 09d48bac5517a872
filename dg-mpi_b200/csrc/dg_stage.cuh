// dg_stage.cuh -- the fused DG stage kernel (sm_100a, FP64).
//
// One launch evaluates, for a batch of E elements per CTA (grid-stride over
// element batches):
//   face traces of the element and of its six neighbours (2D sum-factorised
//   interpolation of boundary coefficient slices; the neighbour read is the
//   on-device periodic face gather that replaces construct_face_states +
//   MemoryNetwork::communicate_face_solution, src/solver/base.cpp:287-327 and
//   src/memory/memory_network.cpp:55-175),
//   the numerical flux at every face point in the reference's L/R convention
//   (flux_functors_impl.h:168-264) with the L=-F / R=+F sign
//   (base.cpp:329-374), the face lift Bf^T F (solver/tools.cpp:38-63),
//   the volume integral: basis->quadrature interpolation, Euler flux,
//   contravariant transform and grad-basis^T contraction
//   (helpers.cpp:185-198, flux_functors_impl.h:46-115, tools.cpp:7-35),
//   the inverse mass (Kronecker product of 1D inverses / det J for affine
//   elements, replacing the dense per-element iMM of tools.cpp:124-139),
//   and the RK4 / forward-Euler stage update (stepper.cpp:23-142).
// Every 3D contraction is sum-factorised into 1D pencil passes through
// shared memory; the last interpolation pass, the pointwise flux and the
// first divergence pass are fused per (x,y) pencil in registers.
#pragma once
#include <cstdint>

#include "dg_physics.cuh"

namespace dgk {

constexpr int kMaxP = 5;
constexpr int kTabB = (kMaxP + 2) * (kMaxP + 1);

// 1D tables per order (filled once per process; see dg_capi.cu)
__constant__ double cB[kMaxP + 1][kTabB];      // B[q*N + b]
__constant__ double cD[kMaxP + 1][kTabB];      // D[q*N + b]
__constant__ double cW[kMaxP + 1][kMaxP + 2];  // GL weights
__constant__ double cMinv[kMaxP + 1][(kMaxP + 1) * (kMaxP + 1)];

struct GeoDev {
    double JD[9];
    double inv_djac;
    double N[6][3];
};

enum StageMode : int {
    kModeResidual = 0,  // out = R(Us)
    kModeMassInv = 1,   // out = dt * M^-1 R(Us)
    kModeRK1 = 2,       // acc = k; out = U0 + k/2
    kModeRK2 = 3,       // acc += 2k; out = U0 + k/2
    kModeRK3 = 4,       // acc += 2k; out = U0 + k
    kModeRK4 = 5,       // out = U0 + (acc + k)/6
    kModeFE = 6         // out = U0 + k
};

enum StatusBits : unsigned {
    kStatusRho = 1u,
    kStatusPressure = 2u,
    kStatusNaN = 4u,
    kStatusHLLC = 8u
};

struct StageArgs {
    const double* Us;       // state the residual is evaluated at, [ne][5][nb]
    const double* U0;       // state at the start of the step, [ne][5][nb]
    double* acc;            // RK4 accumulator, [ne][5][nb]
    double* out;            // output, [ne][5][nb]
    const int2* conn;       // [ne][6]
    const int* geo_class;   // [ne]
    const GeoDev* geo;      // [nclasses]
    const uint8_t* cmap;    // [ncodes][m*m]
    unsigned* status;
    int ne;
    int flux;               // 0 = Lax-Friedrichs, 1 = HLLC
    int mode;
    double gamma;
    double dt;
};

template <int P>
struct Dim {
    static constexpr int N = P + 1;
    static constexpr int M = P + 2;
    static constexpr int NB = N * N * N;
    static constexpr int NF = M * M;
    static constexpr int N2 = N * N;
};

// variable groups of the fused pointwise phase: all five variables at once up
// to p = 3, two groups above (register budget)
template <int P>
struct Groups {
    static constexpr int count = P <= 3 ? 1 : 2;
    static constexpr int first(int g) { return count == 1 ? 0 : (g == 0 ? 0 : 3); }
    static constexpr int size(int g) { return count == 1 ? 5 : (g == 0 ? 3 : 2); }
    static constexpr int max_size = count == 1 ? 5 : 3;
};

template <int P>
struct Work {
    using D = Dim<P>;
    // face phase: own traces [6][5][NF], neighbour traces [6][5][NF], pass buffer [6][5][N*M]
    static constexpr int face = 60 * D::NF + 30 * D::N * D::M;
    // volume phase: X2 [5][N][M][M] first; X1 [5][N][N][M] after it, later
    // overlaid by the divergence buffers A [nv][3][N][M][M] and C [nv][2][N][N][M]
    static constexpr int x2 = 5 * D::N * D::NF;
    static constexpr int x1 = 5 * D::N2 * D::M;
    static constexpr int div = Groups<P>::max_size * (3 * D::N * D::NF + 2 * D::N2 * D::M);
    static constexpr int vol = x2 + (x1 > div ? x1 : div);
    static constexpr int per_elem = face > vol ? face : vol;
};

__device__ __forceinline__ int face_axis(int f) { return f == 2 || f == 4 ? 0 : (f == 1 || f == 3 ? 1 : 2); }
__device__ __forceinline__ int face_side(int f) { return f == 2 || f == 3 || f == 5 ? 1 : 0; }

// coefficient index of boundary-slice entry (b0, b1) of face f
template <int P>
__device__ __forceinline__ int slice_index(int f, int b0, int b1)
{
    constexpr int N = P + 1;
    const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
    if (ax == 0) return b1 * N * N + b0 * N + sidx;
    if (ax == 1) return b1 * N * N + sidx * N + b0;
    return sidx * N * N + b1 * N + b0;
}

template <int P, int E, int NT>
__global__ void __launch_bounds__(NT) stage_kernel(StageArgs a)
{
    using D = Dim<P>;
    constexpr int N = D::N, M = D::M, NB = D::NB, NF = D::NF, N2 = D::N2;
    constexpr int W = Work<P>::per_elem;
    extern __shared__ double smem[];
    double* sU = smem;                  // [E][5][NB]
    double* sRes = sU + E * 5 * NB;     // [E][5][NB]
    double* sW = sRes + E * 5 * NB;     // [E][W]
    const double* __restrict__ Bt = cB[P];
    const double* __restrict__ Dt = cD[P];
    const double* __restrict__ Wt = cW[P];
    const double* __restrict__ Mi = cMinv[P];
    const int tid = threadIdx.x;
    const double gamma = a.gamma;
    unsigned status = 0;

    for (int e0 = blockIdx.x * E; e0 < a.ne; e0 += gridDim.x * E) {
        // ---- load the batch's coefficients (tail elements repeat the last) ----
        for (int i = tid; i < E * 5 * NB; i += NT) {
            const int e = i / (5 * NB), r = i - e * (5 * NB);
            const int ge = min(e0 + e, a.ne - 1);
            sU[i] = a.Us[(size_t)ge * 5 * NB + r];
        }
        __syncthreads();

        // ---- own face traces: slice rows -> [b1][t0] -> [t1][t0] ----
        for (int i = tid; i < E * 30 * N; i += NT) {
            const int b1 = i % N, v = (i / N) % 5, f = (i / (5 * N)) % 6, e = i / (30 * N);
            double row[N];
#pragma unroll
            for (int b0 = 0; b0 < N; ++b0) row[b0] = sU[(e * 5 + v) * NB + slice_index<P>(f, b0, b1)];
            double* T1 = sW + e * W + 60 * NF + ((f * 5 + v) * N + b1) * M;
#pragma unroll
            for (int t = 0; t < M; ++t) {
                double s = 0.0;
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) s += Bt[t * N + b0] * row[b0];
                T1[t] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < E * 30 * M; i += NT) {
            const int t0 = i % M, v = (i / M) % 5, f = (i / (5 * M)) % 6, e = i / (30 * M);
            const double* T1 = sW + e * W + 60 * NF + (f * 5 + v) * N * M;
            double col[N];
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1) col[b1] = T1[b1 * M + t0];
            double* Tr = sW + e * W + (f * 5 + v) * NF;
#pragma unroll
            for (int t1 = 0; t1 < M; ++t1) {
                double s = 0.0;
#pragma unroll
                for (int b1 = 0; b1 < N; ++b1) s += Bt[t1 * N + b1] * col[b1];
                Tr[t1 * M + t0] = s;
            }
        }
        __syncthreads();

        // ---- neighbour traces (periodic face gather) on the neighbour's face ----
        for (int i = tid; i < E * 30 * N; i += NT) {
            const int b1 = i % N, v = (i / N) % 5, f = (i / (5 * N)) % 6, e = i / (30 * N);
            const int ge = min(e0 + e, a.ne - 1);
            const int2 c = a.conn[ge * 6 + f];
            const int fn = c.y & 7;
            double row[N];
            if (c.x >= e0 && c.x < e0 + E) {
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) row[b0] = sU[((c.x - e0) * 5 + v) * NB + slice_index<P>(fn, b0, b1)];
            } else {
                const double* src = a.Us + ((size_t)c.x * 5 + v) * NB;
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) row[b0] = __ldg(src + slice_index<P>(fn, b0, b1));
            }
            double* T1 = sW + e * W + 60 * NF + ((f * 5 + v) * N + b1) * M;
#pragma unroll
            for (int t = 0; t < M; ++t) {
                double s = 0.0;
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) s += Bt[t * N + b0] * row[b0];
                T1[t] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < E * 30 * M; i += NT) {
            const int t0 = i % M, v = (i / M) % 5, f = (i / (5 * M)) % 6, e = i / (30 * M);
            const double* T1 = sW + e * W + 60 * NF + (f * 5 + v) * N * M;
            double col[N];
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1) col[b1] = T1[b1 * M + t0];
            double* Tn = sW + e * W + 30 * NF + (f * 5 + v) * NF;
#pragma unroll
            for (int t1 = 0; t1 < M; ++t1) {
                double s = 0.0;
#pragma unroll
                for (int b1 = 0; b1 < N; ++b1) s += Bt[t1 * N + b1] * col[b1];
                Tn[t1 * M + t0] = s;
            }
        }
        __syncthreads();

        // ---- numerical flux at every face point, written over the own trace ----
        for (int i = tid; i < E * 6 * NF; i += NT) {
            const int cidx = i % NF, f = (i / NF) % 6, e = i / (6 * NF);
            const int ge = min(e0 + e, a.ne - 1);
            const int2 c = a.conn[ge * 6 + f];
            const int fn = c.y & 7, isL = (c.y >> 3) & 1, code = c.y >> 4;
            const int cn = a.cmap[code * NF + cidx];
            double* Tr = sW + e * W + f * 5 * NF;
            const double* Tn = sW + e * W + 30 * NF + f * 5 * NF;
            double Uo[5], Un[5], F[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                Uo[v] = Tr[v * NF + cidx];
                Un[v] = Tn[v * NF + cn];
            }
            const GeoDev* g = a.geo + (isL ? a.geo_class[ge] : a.geo_class[c.x]);
            const int fl = isL ? f : fn;
            const double Nv[3] = {g->N[fl][0], g->N[fl][1], g->N[fl][2]};
            const double* UL = isL ? Uo : Un;
            const double* UR = isL ? Un : Uo;
            if (a.flux == 1) {
                if (!dgp::flux_hllc(gamma, UL, UR, Nv, F)) status |= kStatusHLLC;
            } else {
                dgp::flux_lax_friedrichs(gamma, UL, UR, Nv, F);
            }
            const double w = Wt[cidx % M] * Wt[cidx / M];
            const double sgn = isL ? -1.0 : 1.0;
#pragma unroll
            for (int v = 0; v < 5; ++v) Tr[v * NF + cidx] = sgn * (F[v] * w);
        }
        __syncthreads();

        // ---- face lift: [t1][t0] -> [t1][b0] -> [b1][b0] ----
        for (int i = tid; i < E * 30 * M; i += NT) {
            const int t1 = i % M, v = (i / M) % 5, f = (i / (5 * M)) % 6, e = i / (30 * M);
            const double* Fq = sW + e * W + (f * 5 + v) * NF + t1 * M;
            double row[M];
#pragma unroll
            for (int t0 = 0; t0 < M; ++t0) row[t0] = Fq[t0];
            double* T1 = sW + e * W + 60 * NF + ((f * 5 + v) * M + t1) * N;
#pragma unroll
            for (int b0 = 0; b0 < N; ++b0) {
                double s = 0.0;
#pragma unroll
                for (int t0 = 0; t0 < M; ++t0) s += Bt[t0 * N + b0] * row[t0];
                T1[b0] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < E * 30 * N; i += NT) {
            const int b0 = i % N, v = (i / N) % 5, f = (i / (5 * N)) % 6, e = i / (30 * N);
            const double* T1 = sW + e * W + 60 * NF + (f * 5 + v) * M * N;
            double col[M];
#pragma unroll
            for (int t1 = 0; t1 < M; ++t1) col[t1] = T1[t1 * N + b0];
            double* L = sW + e * W + 30 * NF + (f * 5 + v) * N2;
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1) {
                double s = 0.0;
#pragma unroll
                for (int t1 = 0; t1 < M; ++t1) s += Bt[t1 * N + b1] * col[t1];
                L[b1 * N + b0] = s;
            }
        }
        __syncthreads();
        // gather the six face contributions into the residual
        for (int i = tid; i < E * 5 * NB; i += NT) {
            const int b = i % NB, v = (i / NB) % 5, e = i / (5 * NB);
            const int bc[3] = {b % N, (b / N) % N, b / N2};
            const double* L = sW + e * W + 30 * NF + v * N2;
            double s = 0.0;
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
                if (bc[ax] == sidx) {
                    const int b0 = ax == 0 ? bc[1] : bc[0];
                    const int b1 = ax == 2 ? bc[1] : bc[2];
                    s += L[f * 5 * N2 + b1 * N + b0];
                }
            }
            sRes[i] = s;
        }
        __syncthreads();

        // ---- volume: interpolation passes x, y ----
        double* X2 = sW;                     // per element: [5][N][M][M]
        double* X1 = sW + Work<P>::x2;       // per element: [5][N][N][M]
        for (int i = tid; i < E * 5 * N2; i += NT) {
            const int byz = i % N2, v = (i / N2) % 5, e = i / (5 * N2);
            const double* u = sU + (e * 5 + v) * NB + byz * N;
            double row[N];
#pragma unroll
            for (int bx = 0; bx < N; ++bx) row[bx] = u[bx];
            double* o = X1 + e * W + (v * N2 + byz) * M;
#pragma unroll
            for (int qx = 0; qx < M; ++qx) {
                double s = 0.0;
#pragma unroll
                for (int bx = 0; bx < N; ++bx) s += Bt[qx * N + bx] * row[bx];
                o[qx] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < E * 5 * N * M; i += NT) {
            const int qx = i % M, bz = (i / M) % N, v = (i / (M * N)) % 5, e = i / (5 * N * M);
            const double* x1 = X1 + e * W + (v * N + bz) * N * M;
            double col[N];
#pragma unroll
            for (int by = 0; by < N; ++by) col[by] = x1[by * M + qx];
            double* o = X2 + e * W + (v * N + bz) * NF;
#pragma unroll
            for (int qy = 0; qy < M; ++qy) {
                double s = 0.0;
#pragma unroll
                for (int by = 0; by < N; ++by) s += Bt[qy * N + by] * col[by];
                o[qy * M + qx] = s;
            }
        }
        __syncthreads();

        // ---- fused: z interpolation, Euler flux, contravariant transform,
        //      first (z) divergence contraction; then y and x contractions ----
#pragma unroll
        for (int g = 0; g < Groups<P>::count; ++g) {
            constexpr int GMAX = Groups<P>::max_size;
            const int gv0 = Groups<P>::first(g), gnv = Groups<P>::size(g);
            // A: [nv][3][N][M][M] over X1 ; C: [nv][2][N][N][M] after it
            double* Abuf = sW + Work<P>::x2;
            double* Cbuf = Abuf + GMAX * 3 * N * NF;
            for (int i0 = 0; i0 < E * NF; i0 += NT) {
                const int i = i0 + tid;
                const bool active = i < E * NF;
                const int e = active ? i / NF : 0, qxy = active ? i % NF : 0;
                const int qx = qxy % M, qy = qxy / M;
                double xz[5][N];
                if (active) {
#pragma unroll
                    for (int v = 0; v < 5; ++v)
#pragma unroll
                        for (int bz = 0; bz < N; ++bz) xz[v][bz] = X2[e * W + (v * N + bz) * NF + qxy];
                }
                if (active) {
                    const int ge = min(e0 + e, a.ne - 1);
                    const GeoDev* geo = a.geo + a.geo_class[ge];
                    double JD[9];
#pragma unroll
                    for (int k = 0; k < 9; ++k) JD[k] = geo->JD[k];
                    double acc[GMAX][3][N];
#pragma unroll
                    for (int v = 0; v < GMAX; ++v)
#pragma unroll
                        for (int d = 0; d < 3; ++d)
#pragma unroll
                            for (int bz = 0; bz < N; ++bz) acc[v][d][bz] = 0.0;
                    const double wxy = Wt[qx] * Wt[qy];
#pragma unroll
                    for (int qz = 0; qz < M; ++qz) {
                        double U[5];
#pragma unroll
                        for (int v = 0; v < 5; ++v) {
                            double s = 0.0;
#pragma unroll
                            for (int bz = 0; bz < N; ++bz) s += Bt[qz * N + bz] * xz[v][bz];
                            U[v] = s;
                        }
                        if (g == 0) {
                            const double p = dgp::pressure(gamma, U);
                            if (!(U[0] > 0.0)) status |= kStatusRho;
                            if (!(p > 0.0)) status |= kStatusPressure;
                            if (U[0] != U[0] || p != p) status |= kStatusNaN;
                        }
                        double F[15];
                        dgp::interior_flux(gamma, U, F);
                        const double wq = wxy * Wt[qz];
#pragma unroll
                        for (int vv = 0; vv < GMAX; ++vv) {
                            if (vv < gnv) {
                                const int v = gv0 + vv;
#pragma unroll
                                for (int d = 0; d < 3; ++d) {
                                    const double G = (F[v] * JD[d * 3 + 0] + F[5 + v] * JD[d * 3 + 1] +
                                                      F[10 + v] * JD[d * 3 + 2]) * wq;
#pragma unroll
                                    for (int bz = 0; bz < N; ++bz)
                                        acc[vv][d][bz] += (d == 2 ? Dt[qz * N + bz] : Bt[qz * N + bz]) * G;
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int vv = 0; vv < GMAX; ++vv)
                        if (vv < gnv)
#pragma unroll
                            for (int d = 0; d < 3; ++d)
#pragma unroll
                                for (int bz = 0; bz < N; ++bz)
                                    Abuf[e * W + ((vv * 3 + d) * N + bz) * NF + qxy] = acc[vv][d][bz];
                }
            }
            __syncthreads();
            // y contraction: C0 = By^T A0 ; C12 = Dy^T A1 + By^T A2
            for (int i = tid; i < E * gnv * N * M; i += NT) {
                const int qx = i % M, bz = (i / M) % N, vv = (i / (M * N)) % gnv, e = i / (gnv * N * M);
                const double* A0 = Abuf + e * W + ((vv * 3 + 0) * N + bz) * NF + qx;
                const double* A1 = Abuf + e * W + ((vv * 3 + 1) * N + bz) * NF + qx;
                const double* A2 = Abuf + e * W + ((vv * 3 + 2) * N + bz) * NF + qx;
                double c0[N], c12[N];
#pragma unroll
                for (int by = 0; by < N; ++by) { c0[by] = 0.0; c12[by] = 0.0; }
#pragma unroll
                for (int qy = 0; qy < M; ++qy) {
                    const double a0 = A0[qy * M], a1 = A1[qy * M], a2 = A2[qy * M];
#pragma unroll
                    for (int by = 0; by < N; ++by) {
                        c0[by] += Bt[qy * N + by] * a0;
                        c12[by] += Dt[qy * N + by] * a1 + Bt[qy * N + by] * a2;
                    }
                }
                double* C = Cbuf + e * W + ((vv * 2) * N + bz) * N * M + qx;
#pragma unroll
                for (int by = 0; by < N; ++by) {
                    C[by * M] = c0[by];
                    C[N * N * M + by * M] = c12[by];
                }
            }
            __syncthreads();
            // x contraction into the residual: res += Dx^T C0 + Bx^T C12
            for (int i = tid; i < E * gnv * N2; i += NT) {
                const int byz = i % N2, vv = (i / N2) % gnv, e = i / (gnv * N2);
                const int bz = byz / N, by = byz % N;
                const double* C0 = Cbuf + e * W + ((vv * 2) * N + bz) * N * M + by * M;
                const double* C12 = C0 + N * N * M;
                double r[N];
#pragma unroll
                for (int bx = 0; bx < N; ++bx) r[bx] = 0.0;
#pragma unroll
                for (int qx = 0; qx < M; ++qx) {
                    const double c0 = C0[qx], c12 = C12[qx];
#pragma unroll
                    for (int bx = 0; bx < N; ++bx) r[bx] += Dt[qx * N + bx] * c0 + Bt[qx * N + bx] * c12;
                }
                double* res = sRes + (e * 5 + gv0 + vv) * NB + byz * N;
#pragma unroll
                for (int bx = 0; bx < N; ++bx) res[bx] += r[bx];
            }
            __syncthreads();
        }

        if (a.mode == kModeResidual) {
            for (int i = tid; i < E * 5 * NB; i += NT) {
                const int e = i / (5 * NB);
                if (e0 + e < a.ne) a.out[(size_t)e0 * 5 * NB + i] = sRes[i];
            }
            __syncthreads();
            continue;
        }

        // ---- inverse mass: x and y passes in place, z pass fused with the update ----
        for (int i = tid; i < E * 5 * N2; i += NT) {
            double* r = sRes + i * N;  // pencil along x
            double t[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t[k] = r[k];
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t[k];
                r[j] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < E * 5 * N2; i += NT) {
            const int bx = i % N, bz = (i / N) % N, ev = i / N2;
            double* r = sRes + ev * NB + bz * N2 + bx;  // pencil along y
            double t[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t[k] = r[k * N];
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t[k];
                r[j * N] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < E * 5 * N2; i += NT) {
            const int bxy = i % N2, ev = i / N2, e = ev / 5;
            if (e0 + e >= a.ne) continue;
            const int ge = e0 + e;
            const double scale = a.dt * a.geo[a.geo_class[ge]].inv_djac;
            const double* r = sRes + ev * NB + bxy;  // pencil along z
            double t[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t[k] = r[k * N2];
            const size_t gbase = (size_t)e0 * 5 * NB + (size_t)ev * NB + bxy;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t[k];
                const double kk = scale * s;
                const size_t gi = gbase + (size_t)j * N2;
                switch (a.mode) {
                    case kModeMassInv: a.out[gi] = kk; break;
                    case kModeRK1: a.acc[gi] = kk; a.out[gi] = 0.5 * kk + a.U0[gi]; break;
                    case kModeRK2: a.acc[gi] = a.acc[gi] + 2.0 * kk; a.out[gi] = 0.5 * kk + a.U0[gi]; break;
                    case kModeRK3: a.acc[gi] = a.acc[gi] + 2.0 * kk; a.out[gi] = 1.0 * kk + a.U0[gi]; break;
                    case kModeRK4: a.out[gi] = a.U0[gi] + (1.0 / 6.0) * (a.acc[gi] + kk); break;
                    default: a.out[gi] = a.U0[gi] + 1.0 * kk; break;
                }
            }
        }
        __syncthreads();
    }
    if (status) atomicOr(a.status, status);
}

template <int P, int E>
constexpr size_t stage_smem_bytes()
{
    return sizeof(double) * (size_t)E * (10 * Dim<P>::NB + Work<P>::per_elem);
}

}  // namespace dgk
