// dg_stage.cuh -- the DG stage kernel and the face-flux kernel (sm_100a; FP64, or FP32 residual with FP64 state).
//
// One launch evaluates, for batches of E elements per CTA (grid-stride):
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
//   elements, replacing the dense per-element iMM of tools.cpp:124-139; the
//   dense per-element inverse itself on general trilinear elements),
//   and the RK4 / forward-Euler stage update (stepper.cpp:23-142).
// With the face-flux launch option a second kernel, face_flux_kernel, runs
// before it and computes the traces and the flux of every face once; the
// stage kernel then stages its six faces' fluxes instead.
//
// Every 3D contraction is sum-factorised into 1D passes over shared memory:
// either the last interpolation pass, the pointwise flux and the first
// divergence pass fused per (x,y) pencil in registers, or (unfused volume)
// separate passes over a point array holding every quadrature point; traces
// and lifts are 2D interpolations per (element, face, variable) or per output
// row.  Shared strides, task orders and (at p = 3) a row rotation of the
// coefficient blocks are chosen against bank conflicts (see qs_stride,
// TaskOrd and Lay::cw).  The coefficients of the next batch are prefetched
// with cp.async while the current batch computes.
#pragma once
#include <cstdint>
#include <type_traits>
#include <vector>

#include "dg_physics.cuh"

namespace dgk {

constexpr int kMaxP = 5;
constexpr int kTabB = (kMaxP + 2) * (kMaxP + 1);

// 1D tables of the case's order, passed in the kernel's parameter block (it
// lives in the constant bank, so the unrolled loops read them as constant
// operands); see dgh::make_tables
struct StageTables {
    double B[kTabB];                           // B[q*N + b]: basis at the GL points
    double D[kTabB];                           // D[q*N + b]: its derivative
    double W[kMaxP + 2];                       // GL weights
    double Minv[(kMaxP + 1) * (kMaxP + 1)];    // inverse 1D mass matrix (always FP64)
    float Bf[kTabB];                           // FP32 copies for the mixed-precision residual
    float Df[kTabB];
    float Wf[kMaxP + 2];
    // derivative of the 1D Lagrange basis at its own equidistant nodes,
    // Dn[i*N + j] = l_j'(xi_i) (the tensor-core kernel's nodal derivative)
    float Dn[(kMaxP + 1) * (kMaxP + 1)];
};

template <typename T> struct TabSel;
template <> struct TabSel<double> {
    static __device__ __forceinline__ const double* B(const StageTables& t) { return t.B; }
    static __device__ __forceinline__ const double* D(const StageTables& t) { return t.D; }
    static __device__ __forceinline__ const double* W(const StageTables& t) { return t.W; }
};
template <> struct TabSel<float> {
    static __device__ __forceinline__ const float* B(const StageTables& t) { return t.Bf; }
    static __device__ __forceinline__ const float* D(const StageTables& t) { return t.Df; }
    static __device__ __forceinline__ const float* W(const StageTables& t) { return t.Wf; }
};

struct GeoDev {
    double JD[9];
    double inv_djac;
    double dtf;           // time-step factor: the stage update scales by dt * dtf (1, or a case's dt in a batch)
    double eref;          // FP32 residual: energy reference E_ref (state energy enters as rE - E_ref); 0 for FP64
    double N[6][3];
    double nmag[6];       // |N| per face
    double nhat[6][3];    // N / |N| (Lax-Friedrichs)
    double nunit[6][3];   // N * (1/|N|) (HLLC)
};

// One face of an owned element, built at context creation and prefetched with
// the element's coefficients (48 bytes): the neighbour, the packed neighbour
// face | left role << 3 | permutation code << 4 (as conn), the left element's
// normal data (N/|N| for Lax-Friedrichs, N*(1/|N|) for HLLC, and |N|), the
// element's own geometry class, and (launch option FX) the face's number in
// the face list | 1 << 30 when the flux is stored in this side's point order.
struct FaceRec {
    double n[3];
    double nmag;
    int nbr;
    int info;
    int cls;
    int pad;
};
static_assert(sizeof(FaceRec) == 48, "FaceRec is six 8-byte words");

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
    const FaceRec* frec;    // [ne][6]
    const int* geo_class;   // [ne]
    const GeoDev* geo;      // [nclasses]
    const uint8_t* cmap;    // [ncodes][m*m]
    // general (trilinear) geometry, launch option GE: per element ijac * djac
    // at the volume points [ne][9][(p+2)^3], the face normal data at the own
    // face points [ne][6][4][(p+2)^2] (n as for FaceRec, then |N|), and the
    // inverse mass matrix transposed [ne][nb][nb]
    const double* gjd;
    const double* gnrm;
    const double* gimm;
    // GE with the FP32 residual: the residual of a uniform state at rest with
    // unit pressure [ne][5][nb] (FP64).  The FP32 residual leaves the constant
    // pressure (gamma-1) E_ref out of the momentum fluxes; on affine meshes its
    // volume and face terms cancel, on general meshes the reference's face
    // normals (taken at reference face 0's points) leave a remainder, linear
    // in the pressure, that this table restores.
    const double* gfsd;
    // launch option FX: the faces as (element, face) of the side whose point
    // order the flux is stored in [nface], the range [face_begin, nface) one
    // face-kernel launch computes, and the fluxes [nface][5][(p+2)^2] (T
    // values, weights applied, unsigned)
    const int2* faces;
    int face_begin, nface;
    void* fflux;
    int fstride;            // elements per face in fflux: 5 (p+2)^2, or padded to a 16-byte multiple (TC)
    // tensor-core kernel: the basis operator B[q][b] as three BF16 parts in its
    // shared-memory layout (dgk::tc_operator_table)
    const uint16_t* tcop;
    unsigned* status;
    int e_begin, ne;        // the launch computes elements [e_begin, ne)
    int flux;               // 0 = Lax-Friedrichs, 1 = HLLC
    int mode;
    double gamma;
    double dt;
    StageTables tab;
};

__host__ __device__ constexpr int odd(int x) { return x | 1; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Shared-memory bank layout. A warp's FP64 access is served per half-warp
// (16 lanes, bank pair = word % 16), an FP32 access per warp (bank = word % 32);
// distinct words on one bank cost one wavefront each. The point-array row
// stride and the task order of every pass below were chosen together by
// counting the wavefronts of each pass's addresses over all strides up to 16
// past the block size and all task orders (per order and arithmetic width);
// tests/bank_model.py reproduces them. The update pass keeps
// its z-pencil order (consecutive threads write consecutive global words).
//
// point-array row stride of the unfused volume
__host__ __device__ constexpr int qs_stride(int P, int bytes)
{
    return P == 2 ? 79
         : P == 3 ? (bytes == 8 ? 127 : 126)
         : P == 4 ? (bytes == 8 ? 223 : 231)
         : P == 5 ? (bytes == 8 ? 349 : 343)
                  : odd((P + 2) * (P + 2) * (P + 2));
}
// Task orders. Two coordinates: 0 = the first one varies fastest, 1 = the
// second. Three coordinates (c0, c1, c2): O = f + 3 m + 9 s names the fastest,
// middle and slowest one.
template <int P, int BYTES>
struct TaskOrd {
    static constexpr bool W8 = BYTES == 8;
    static constexpr int x = P >= 3 || (P == 2 && !W8) ? 1 : 0;                                 // (v, byz)
    static constexpr int y = P == 2 ? 11 : P == 3 ? 5 : P == 4 ? (W8 ? 5 : 21) : P == 5 ? (W8 ? 21 : 11) : 21;  // (v, qx, bz)
    static constexpr int z = P == 5 && W8 ? 1 : 0;                                              // (qxy, v)
    static constexpr int zc = P == 2 ? (W8 ? 0 : 1) : P == 3 ? 1 : P == 4 ? (W8 ? 1 : 0) : 0;  // (qxy, v)
    static constexpr int yc = P == 2 ? (W8 ? 21 : 11) : P == 3 ? (W8 ? 21 : 5) : P == 4 ? (W8 ? 21 : 11)
                            : P == 5 ? (W8 ? 19 : 21) : 7;                                      // (v, qx, bz)
    static constexpr int xc = P >= 3 || (P == 2 && !W8) ? 1 : 0;                                // (v, byz)
    static constexpr int gather = P == 4 ? 1 : 0;                                               // (b, v)
    static constexpr int minvx = P >= 2 ? 1 : 0;                                                // (v, byz)
    static constexpr int minvy = P == 2 || P == 4 ? 11 : P == 3 || P == 5 ? 7 : 21;             // (v, bx, bz)
    static constexpr int minvxg = P == 5 && W8 ? 0 : 1;                                         // (v, byz), MG
};
template <int O, int n0, int n1>
__device__ __forceinline__ void task2(int r, int& c0, int& c1)
{
    if constexpr (O == 0) {
        c0 = r % n0;
        c1 = r / n0;
    } else {
        c1 = r % n1;
        c0 = r / n1;
    }
}
template <int O, int n0, int n1, int n2>
__device__ __forceinline__ void task3(int r, int& c0, int& c1, int& c2)
{
    constexpr int f = O % 3, m = (O / 3) % 3, s = O / 9;
    static_assert(f != m && m != s && f != s, "task order must name three coordinates");
    constexpr int n[3] = {n0, n1, n2};
    constexpr int nf = n[f], nm = n[m];
    int c[3];
    c[f] = r % nf;
    c[m] = (r / nf) % nm;
    c[s] = r / (nf * nm);
    c0 = c[0];
    c1 = c[1];
    c2 = c[2];
}

// G = number of variable groups of the fused pointwise phase (register budget);
// T = arithmetic of the residual (the work area W holds T values, everything
// else FP64); FL: launch options, flag 1 (PZ) -- the groups' pencil tasks run in
// one phase (the z-contraction output of all five variables is held at once);
// flag 2 (SB) -- one coefficient buffer, refilled with the next batch once the
// traces have read it (instead of two); flag 4 (UF) -- unfused volume: the z
// interpolation, the pointwise flux and each contraction are separate passes
// over a point array holding all quadrature points (the flux is evaluated once
// per point instead of once per variable group; G is unused); flag 8 (RS) --
// traces and lifts as one task per output row instead of per face slice;
// flag 16 (K1) -- one face-flux point per thread and iteration (registers);
// flag 32 (GE) -- general (trilinear) geometry: per-point metric terms and
// normals and a dense per-element inverse mass matrix, read from global
// memory (requires UF); flag 64 (FX) -- face fluxes from the face kernel:
// every interior face's flux is computed once (face_flux_kernel, launched
// before the stage kernel) and each element stages its six faces' fluxes
// instead of computing traces and fluxes (requires SB); flag 4096 (MG) -- the
// six faces' lifted fluxes added to the residual inside the inverse mass's x
// pass instead of a separate pass over the residual (affine geometry)
template <int P, int G, typename T = double, int FL = 0>
struct Lay {
    static constexpr bool PZ = FL & 1, SB = FL & 2, UF = FL & 4, RS = FL & 8, K1 = FL & 16, GE = FL & 32, FX = FL & 64;
    static constexpr bool MG = FL & 4096;
    static_assert(!GE || UF, "general geometry needs the unfused volume");
    static_assert(!FX || SB, "face fluxes from the face kernel need the single buffer");
    static_assert(!MG || !GE, "the folded lift gather needs the Kronecker inverse mass");
    static constexpr int N = P + 1, M = P + 2, NB = N * N * N, NF = M * M, N2 = N * N;
    static constexpr int GV = G == 1 ? 5 : (G == 2 ? 3 : 2);  // variables per group (max)
    static constexpr int GA = PZ ? 5 : GV;       // variables of the z-contraction buffers
    static constexpr int VS = odd(NB);           // per-variable stride of U / residual
    static constexpr int ES = 5 * VS;            // per-element stride of U / residual
    static constexpr int FS = odd(NF);           // per-(face, variable) stride of traces
    static constexpr int NS = odd(N2);           // per-(face, variable) stride of neighbour slices
    static constexpr int X1S = odd(N2 * M);      // [bz][by][qx] block
    static constexpr int X2S = odd(N * NF);      // [bz][qy][qx] block
    static constexpr int QS = qs_stride(P, sizeof(T));  // [qz][qy][qx] block of the point array (UF)
    // word of coefficient (bx, by, bz) in a variable's block of U / residual /
    // U0 / accumulator: at p = 3 the rows are rotated so that every axis-aligned
    // plane of the 4x4x4 block falls on 16 distinct bank pairs (the x, y and z
    // pencils of a variable, 16 to a half-warp, are then conflict-free);
    // otherwise x fastest
    static constexpr bool SWZ = N == 4;
    __host__ __device__ static constexpr int cw(int bx, int by, int bz)
    {
        return SWZ ? 16 * by + 4 * ((bx + by) & 3) + ((bz + bx) & 3) : (bz * N + by) * N + bx;
    }
    __host__ __device__ static constexpr int cwl(int b) { return SWZ ? cw(b % N, (b / N) % N, b / N2) : b; }
    // cw is a bijection of the block onto words 0 .. NB-1 and, rotated, every
    // axis-aligned plane covers all 16 bank pairs
    static constexpr bool cw_ok()
    {
        bool word[NB] = {};
        for (int b = 0; b < NB; ++b) {
            const int w = cwl(b);
            if (w < 0 || w >= NB || word[w]) return false;
            word[w] = true;
        }
        if (SWZ)
            for (int ax = 0; ax < 3; ++ax)
                for (int k = 0; k < N; ++k) {
                    bool bank[16] = {};
                    for (int i = 0; i < N; ++i)
                        for (int j = 0; j < N; ++j) {
                            const int w = ax == 0 ? cw(k, i, j) : (ax == 1 ? cw(i, k, j) : cw(i, j, k));
                            if (bank[w % 16]) return false;
                            bank[w % 16] = true;
                        }
                }
        return true;
    }
    static_assert(cw_ok(), "coefficient block layout must be a bijection (and plane-conflict-free when rotated)");
    // per-element work area: face phase {Tr[6][5], Tn[6][5]} x FS;
    // volume phase X2[5] | (X1[5] or A[GA][3] + C[GA][2]), or with UF the
    // point array Q[15] (X2 in its first five rows, X1 after them)
    static constexpr int face = 60 * FS;
    static constexpr int vol =
        UF ? cmax(15 * QS, 5 * QS + 5 * X1S) : 5 * X2S + cmax(5 * X1S, GA * (3 * X2S + 2 * X1S));
    static constexpr int W = odd(cmax(face, vol));
    // FP64 operand region: first the neighbours' boundary slices [30][NS]
    // (with FX: the six faces' fluxes [30][FS] in T), streamed in during the
    // volume phase, then the batch's U0 and RK accumulator [2][ES]
    static constexpr int OPS = cmax(2 * ES, FX ? (30 * FS * (int)sizeof(T) + 7) / 8 : 30 * NS);
    // FP64: U (double-buffered prefetch, or single with SB), residual, operand region
    static constexpr int per_elem_f64 = (SB ? 1 : 2) * ES + ES + OPS;
    // bytes per element, work area in T
    static constexpr size_t bytes_per_elem = sizeof(double) * per_elem_f64 + sizeof(T) * W;
    // face data of a batch: the six face records (the next batch's are
    // prefetched once the flux phase has read them), the element's geometry
    // class and the faces' rows of the face-point permutation
    static constexpr size_t meta_bytes_per_elem = 6 * sizeof(FaceRec) + sizeof(int) + 6 * NF;
};

template <int P, int G>
__host__ __device__ constexpr int group_first(int g)
{
    return G == 1 ? 0 : (G == 2 ? (g == 0 ? 0 : 3) : (g == 0 ? 0 : (g == 1 ? 2 : 4)));
}
template <int P, int G>
__host__ __device__ constexpr int group_size(int g)
{
    return G == 1 ? 5 : (G == 2 ? (g == 0 ? 3 : 2) : (g == 2 ? 1 : 2));
}

// calls f(std::integral_constant<int, I>) for I = I0 .. I1-1
template <int I0, int I1, typename F>
__device__ __forceinline__ void static_for(F&& f)
{
    if constexpr (I0 < I1) {
        f(std::integral_constant<int, I0>{});
        static_for<I0 + 1, I1>(f);
    }
}

__device__ __forceinline__ int face_axis(int f) { return f == 2 || f == 4 ? 0 : (f == 1 || f == 3 ? 1 : 2); }
__device__ __forceinline__ int face_side(int f) { return f == 2 || f == 3 || f == 5 ? 1 : 0; }

// coefficient index (unpadded, x fastest) of boundary-slice entry (b0, b1) of face f
template <int N>
__device__ __forceinline__ int slice_index(int f, int b0, int b1)
{
    const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
    if (ax == 0) return b1 * N * N + b0 * N + sidx;
    if (ax == 1) return b1 * N * N + sidx * N + b0;
    return sidx * N * N + b1 * N + b0;
}

__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gmem_src)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gmem_src)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_t(double* d, const double* g) { cp_async8(d, g); }
__device__ __forceinline__ void cp_async_t(float* d, const float* g) { cp_async4(d, g); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// all but the most recent group complete
__device__ __forceinline__ void cp_async_wait_older() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// queue the face records of batch e0 into dst [E][6]
template <int E, int NT>
__device__ __forceinline__ void prefetch_recs(const FaceRec* __restrict__ frec, int ne, int e0, FaceRec* dst)
{
    constexpr int W8 = 6 * sizeof(FaceRec) / 8;  // 8-byte words per element
    for (int i = threadIdx.x; i < E * W8; i += NT) {
        const int e = i / W8, r = i - e * W8;
        const int ge = min(e0 + e, ne - 1);
        cp_async8(reinterpret_cast<double*>(dst + e * 6) + r, reinterpret_cast<const double*>(frec + (size_t)ge * 6) + r);
    }
}

// queue the coefficients of batch e0 of a global state into the padded
// buffer dst (element stride estride)
template <int P, int G, int E, int NT>
__device__ __forceinline__ void prefetch_batch(const double* __restrict__ Us, int ne, int e0, double* dst,
                                               int estride)
{
    using L = Lay<P, G>;
    for (int i = threadIdx.x; i < E * 5 * L::NB; i += NT) {
        const int e = i / (5 * L::NB), r = i - e * (5 * L::NB), v = r / L::NB, b = r - v * L::NB;
        const int ge = min(e0 + e, ne - 1);
        cp_async8(dst + e * estride + v * L::VS + L::cwl(b), Us + (size_t)ge * 5 * L::NB + r);
    }
}

// The numerical flux at one face point from the left and right states and
// the left element's normal data nd = (n, |N|) (flux_functors_impl.h:168-264):
// HLLC (euler/functions.cpp:298-399) or Lax-Friedrichs (base/functions.cpp:33-89).
// With SHIFT (the FP32 residual) the states carry rE - eref and the constant
// pressure (gamma-1) eref is left out of the momentum fluxes.
template <typename T, bool SHIFT>
__device__ __forceinline__ void numerical_flux(int flux, double gamma_d, T (&UL)[5], T (&UR)[5], const T (&nd)[4],
                                               double eref, T (&Fo)[5], unsigned& status)
{
    const T gamma = T(gamma_d);
    const T nmag = nd[3];
    if (flux == 1) {
        const T nu[3] = {nd[0], nd[1], nd[2]};
        // the FP32 residual keeps the shifted energy and leaves the constant
        // pressure out of the momenta (dgp::flux_hllc_shift)
        const bool ok = SHIFT ? dgp::flux_hllc_shift(gamma, UL, UR, nu, nmag, T(eref), Fo)
                              : dgp::flux_hllc_n(gamma, UL, UR, nu, nmag, Fo);
        if (!ok) status |= kStatusHLLC;
    } else {
        const T nh[3] = {nd[0], nd[1], nd[2]};
        dgp::flux_lax_friedrichs_fast<T, SHIFT>(gamma, UL, UR, nh, nmag, Fo, T(gamma_d * eref), T((gamma_d - 1.0) * eref));
    }
}

// 2D interpolation of an N x N slice s[b1][b0] to the M x M face grid,
// written to out[t1*M + t0]
template <int N, int M, typename T>
__device__ __forceinline__ void interp2d(const T* __restrict__ Bt, const T (&s)[N][N], T* out)
{
    T tmp[N][M];
#pragma unroll
    for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
        for (int t0 = 0; t0 < M; ++t0) {
            T a = T(0);
#pragma unroll
            for (int b0 = 0; b0 < N; ++b0) a += Bt[t0 * N + b0] * s[b1][b0];
            tmp[b1][t0] = a;
        }
#pragma unroll
    for (int t1 = 0; t1 < M; ++t1)
#pragma unroll
        for (int t0 = 0; t0 < M; ++t0) {
            T a = T(0);
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1) a += Bt[t1 * N + b1] * tmp[b1][t0];
            out[t1 * M + t0] = a;
        }
}

// bid / nblk: this block's index among the nblk blocks that share the
// launch's element range (blockIdx.x / gridDim.x).  With a work counter
// (work != nullptr, an ensemble launch) the batches are claimed instead:
// batch k = atomicAdd(work, 1) starts at e_begin + k E, claimed one batch
// ahead by thread 0 and passed on through the two shared slots `slots`, so
// the next batch is known when its prefetch is issued.
template <int P, int E, int NT, int G, typename T, int FL>
__device__ __forceinline__ void stage_body(const StageArgs& a, int bid, int nblk, int* work = nullptr,
                                           int* slots = nullptr)
{
    using L = Lay<P, G, T, FL>;
    constexpr bool PZ = L::PZ, SB = L::SB;
    constexpr int N = L::N, M = L::M, NB = L::NB, NF = L::NF, N2 = L::N2;
    constexpr int VS = L::VS, ES = L::ES, FS = L::FS, NS = L::NS, X1S = L::X1S, X2S = L::X2S, W = L::W, GV = L::GV;
    constexpr int OPS = L::OPS;
    using TO = TaskOrd<P, sizeof(T)>;
    extern __shared__ double smem[];
    double* sUbuf = smem;                  // [2][E][ES] ([1][E][ES] with SB)
    double* sRes = sUbuf + (SB ? 1 : 2) * E * ES;  // [E][ES]
    double* sOps = sRes + E * ES;          // [E][OPS] neighbour slices, then U0 | acc
    T* sW = reinterpret_cast<T*>(sOps + E * OPS);  // [E][W] in the residual's arithmetic
    // face data (see Lay::meta_bytes_per_elem), 16-byte aligned after sW
    unsigned char* meta = reinterpret_cast<unsigned char*>(smem) + ((E * L::bytes_per_elem + 15) / 16) * 16;
    FaceRec* sRec = reinterpret_cast<FaceRec*>(meta);                 // [E][6] this batch's face records
    int* sCls = reinterpret_cast<int*>(sRec + E * 6);                  // [E] geometry classes
    unsigned char* sCm = reinterpret_cast<unsigned char*>(sCls + E);  // [E*6][NF]
    const bool need_u0_acc = a.mode == kModeRK2 || a.mode == kModeRK3 || a.mode == kModeRK4;
    // with SB the coefficient buffer is refilled before the update, so the
    // update's step-start state comes from the operand region in every mode
    const bool stage_u0 = need_u0_acc || (SB && (a.mode == kModeRK1 || a.mode == kModeFE));
    const T* __restrict__ Bt = TabSel<T>::B(a.tab);
    const T* __restrict__ Dt = TabSel<T>::D(a.tab);
    const T* __restrict__ Wt = TabSel<T>::W(a.tab);
    const double* __restrict__ Mi = a.tab.Minv;
    const int tid = threadIdx.x;
    const T gamma = T(a.gamma);
    // the FP32 residual works on rE - E_ref (see dgp::interior_flux_r1)
    constexpr bool kShift = sizeof(T) == 4;
    // face-flux points per thread and iteration: measured best 3 at p = 2 and
    // p = 5, 2 at the other orders (more points add registers); 1 with K1
    constexpr int kFluxPoints = L::K1 ? 1 : ((P == 2 || P == 5) ? 3 : 2);
    unsigned status = 0;
    const int stride = nblk * E;
    int e_first = a.e_begin + bid * E;
    if (work) {
        if (tid == 0) {
            slots[0] = a.e_begin + atomicAdd(work, 1) * E;
            slots[1] = a.e_begin + atomicAdd(work, 1) * E;
        }
        __syncthreads();
        e_first = slots[0];
    }

    int buf = 0;
    if (e_first < a.ne) {
        prefetch_batch<P, G, E, NT>(a.Us, a.ne, e_first, sUbuf, ES);
        prefetch_recs<E, NT>(a.frec, a.ne, e_first, sRec);
    }
    cp_async_commit();

    int en = e_first, it = 0;  // the next batch
    for (int e0 = e_first; e0 < a.ne; e0 = en, buf ^= 1, ++it) {
        double* sU = sUbuf + (SB ? 0 : buf) * E * ES;
        cp_async_wait_all();
        __syncthreads();
        if (work) {
            en = slots[(it + 1) & 1];
            if (tid == 0) slots[it & 1] = a.e_begin + atomicAdd(work, 1) * E;  // read two iterations ago
        } else {
            en = e0 + stride;
        }
        // stream in the neighbours' boundary slices (the periodic face gather)
        // for the face phase, then the next batch's coefficients; one task per
        // (element, face, variable), or per slice row when the CTA has threads
        // to spare
        if constexpr (L::FX) {
            // the six faces' fluxes, computed once per face by the face kernel:
            // the side the flux was computed for reads it in its own point
            // order, the other through the face-point permutation (the lift
            // applies the sign of the element's side)
            const T* gF = reinterpret_cast<const T*>(a.fflux);
            for (int t = tid; t < E * 6 * NF; t += NT) {
                const int c = t % NF, f = (t / NF) % 6, e = t / (6 * NF);
                const FaceRec& rec = sRec[e * 6 + f];
                const int pc = ((rec.pad >> 30) & 1) ? c : a.cmap[(rec.info >> 4) * NF + c];
                const T* src = gF + (size_t)(rec.pad & 0x3fffffff) * a.fstride + pc;
                T* dst = reinterpret_cast<T*>(sOps + e * OPS) + f * 5 * FS + c;
#pragma unroll
                for (int v = 0; v < 5; ++v) cp_async_t(dst + v * FS, src + v * NF);
            }
            for (int e = tid; e < E; e += NT) sCls[e] = sRec[e * 6].cls;
        } else {
            constexpr int kSliceRows = NT > E * 30 ? N : 1;
            for (int t = tid; t < E * 30 * kSliceRows; t += NT) {
                const int row = t % kSliceRows, fv = (t / kSliceRows) % 30, e = t / (30 * kSliceRows);
                const int v = fv % 5, f = fv / 5;
                const FaceRec& rec = sRec[e * 6 + f];
                const int2 c = make_int2(rec.nbr, rec.info);
                const double* src = a.Us + ((size_t)c.x * 5 + v) * NB;
                double* dst = sOps + e * OPS + fv * NS;
#pragma unroll
                for (int r = 0; r < N / kSliceRows; ++r) {
                    const int b1 = row + r;
#pragma unroll
                    for (int b0 = 0; b0 < N; ++b0) cp_async8(dst + b1 * N + b0, src + slice_index<N>(c.y & 7, b0, b1));
                }
                // this face's row of the face-point permutation, shared out over the face's tasks
                const int fm = e * 6 + f, code = c.y >> 4;
                for (int q = v * kSliceRows + row; q < NF; q += 5 * kSliceRows) sCm[fm * NF + q] = a.cmap[code * NF + q];
                if (fv == 0 && row == 0) sCls[e] = rec.cls;
            }
        }
        cp_async_commit();
        if (!SB && en < a.ne)
            prefetch_batch<P, G, E, NT>(a.Us, a.ne, en, sUbuf + (buf ^ 1) * E * ES, ES);
        cp_async_commit();

        // ---- volume: interpolation passes x, y ----
        // per element: X2 [5][X2V] with [bz][qy][qx] (with UF, the first five
        // rows of the point array, where the z pass interpolates in place) and
        // X1 [5][X1S] with [bz][by][qx] (with UF, in rows 5.. of the point array)
        constexpr int X2V = L::UF ? L::QS : X2S;
        T* X2 = sW;
        T* X1 = sW + 5 * X2V;
        for (int i = tid; i < E * 5 * N2; i += NT) {
            const int e = i / (5 * N2);
            int v, byz;
            task2<TO::x, 5, N2>(i - e * 5 * N2, v, byz);
            const double* u = sU + e * ES + v * VS;
            const int by = byz % N, bz = byz / N;
            const double sh = kShift && v == 4 ? a.geo[sRec[e * 6].cls].eref : 0.0;
            T row[N];
#pragma unroll
            for (int bx = 0; bx < N; ++bx) {
                const double ub = u[L::cw(bx, by, bz)];
                row[bx] = kShift ? T(ub - sh) : T(ub);
            }
            T* o = X1 + e * W + v * X1S + byz * M;
#pragma unroll
            for (int qx = 0; qx < M; ++qx) {
                T s = T(0);
#pragma unroll
                for (int bx = 0; bx < N; ++bx) s += Bt[qx * N + bx] * row[bx];
                o[qx] = s;
            }
        }
        __syncthreads();
        // with FX the x pass was the coefficients' last reader: refill the
        // single buffer with the next batch now
        if constexpr (L::FX) {
            if (en < a.ne) prefetch_batch<P, G, E, NT>(a.Us, a.ne, en, sU, ES);
            cp_async_commit();
        }
        for (int i = tid; i < E * 5 * N * M; i += NT) {
            const int e = i / (5 * N * M);
            int v, qx, bz;
            task3<TO::y, 5, M, N>(i - e * 5 * N * M, v, qx, bz);
            const T* x1 = X1 + e * W + v * X1S + bz * N * M + qx;
            T col[N];
#pragma unroll
            for (int by = 0; by < N; ++by) col[by] = x1[by * M];
            T* o = X2 + e * W + v * X2V + bz * NF + qx;
#pragma unroll
            for (int qy = 0; qy < M; ++qy) {
                T s = T(0);
#pragma unroll
                for (int by = 0; by < N; ++by) s += Bt[qy * N + by] * col[by];
                o[qy * M] = s;
            }
        }
        __syncthreads();

        if constexpr (L::UF) {
            // ---- unfused: z interpolation in the point array, the flux at
            //      every point, then z, y and x contractions (in place) ----
            constexpr int QS = L::QS, NQ = M * NF;
            T* Q = sW;  // per element: [15][QS], point index qz*NF + qy*M + qx
            // z interpolation in place: each task owns one (variable, x-y point) column
            for (int i = tid; i < E * 5 * NF; i += NT) {
                const int e = i / (5 * NF);
                int qxy, v;
                task2<TO::z, NF, 5>(i - e * 5 * NF, qxy, v);
                T* o = Q + e * W + v * QS + qxy;
                T col[N];
#pragma unroll
                for (int bz = 0; bz < N; ++bz) col[bz] = o[bz * NF];
#pragma unroll
                for (int qz = 0; qz < M; ++qz) {
                    T s = T(0);
#pragma unroll
                    for (int bz = 0; bz < N; ++bz) s += Bt[qz * N + bz] * col[bz];
                    o[qz * NF] = s;
                }
            }
            __syncthreads();
            // Euler flux and contravariant transform: point q's five states become
            // its fifteen components (v, d) in row 3v+d (each thread owns column q)
            for (int i = tid; i < E * NQ; i += NT) {
                const int q = i % NQ, e = i / NQ;
                const int qx = q % M, qy = (q / M) % M, qz = q / NF;
                T* qp = Q + e * W + q;
                T U[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) U[v] = qp[v * QS];
                const GeoDev* geo = a.geo + sCls[e];
                const T hr = kShift ? T(a.gamma * geo->eref) : T(0);
                const T pref = kShift ? T((a.gamma - 1.0) * geo->eref) : T(0);
                T F[15];
                const T p = dgp::interior_flux_r1<T, kShift>(gamma, U, F, hr);
                if (!(U[0] > T(0))) status |= kStatusRho;
                if (!(p + pref > T(0))) status |= kStatusPressure;
                if (U[0] != U[0] || p != p) status |= kStatusNaN;
                T JD[9];
                if constexpr (L::GE) {
                    const double* gj = a.gjd + (size_t)min(e0 + e, a.ne - 1) * 9 * NQ + q;
#pragma unroll
                    for (int k = 0; k < 9; ++k) JD[k] = T(gj[(size_t)k * NQ]);
                } else {
#pragma unroll
                    for (int k = 0; k < 9; ++k) JD[k] = T(geo->JD[k]);
                }
                const T wq = Wt[qx] * Wt[qy] * Wt[qz];
#pragma unroll
                for (int v = 0; v < 5; ++v)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        qp[(v * 3 + d) * QS] = (F[v] * JD[d * 3 + 0] + F[5 + v] * JD[d * 3 + 1] + F[10 + v] * JD[d * 3 + 2]) * wq;
            }
            __syncthreads();
            // z contraction per (variable, x-y point), the three directions together:
            // A_d = Bz^T G_d (d = 0, 1), A_2 = Dz^T G_2, written over the column
            for (int i = tid; i < E * 5 * NF; i += NT) {
                const int e = i / (5 * NF);
                int qxy, v;
                task2<TO::zc, NF, 5>(i - e * 5 * NF, qxy, v);
                T* g = Q + e * W + (v * 3) * QS + qxy;
                T a0[N], a1[N], a2[N];
#pragma unroll
                for (int bz = 0; bz < N; ++bz) { a0[bz] = T(0); a1[bz] = T(0); a2[bz] = T(0); }
#pragma unroll
                for (int qz = 0; qz < M; ++qz) {
                    const T g0 = g[qz * NF], g1 = g[QS + qz * NF], g2 = g[2 * QS + qz * NF];
#pragma unroll
                    for (int bz = 0; bz < N; ++bz) {
                        a0[bz] += Bt[qz * N + bz] * g0;
                        a1[bz] += Bt[qz * N + bz] * g1;
                        a2[bz] += Dt[qz * N + bz] * g2;
                    }
                }
#pragma unroll
                for (int bz = 0; bz < N; ++bz) {
                    g[bz * NF] = a0[bz];
                    g[QS + bz * NF] = a1[bz];
                    g[2 * QS + bz * NF] = a2[bz];
                }
            }
            __syncthreads();
            // y contraction per (variable, bz, qx): C0 = By^T A0 into row 3v,
            // C12 = Dy^T A1 + By^T A2 into row 3v+1
            for (int i = tid; i < E * 5 * N * M; i += NT) {
                const int e = i / (5 * N * M);
                int v, qx, bz;
                task3<TO::yc, 5, M, N>(i - e * 5 * N * M, v, qx, bz);
                T* A0 = Q + e * W + (v * 3) * QS + bz * NF + qx;
                const T* A1 = A0 + QS;
                const T* A2 = A1 + QS;
                T c0[N], c12[N];
#pragma unroll
                for (int by = 0; by < N; ++by) { c0[by] = T(0); c12[by] = T(0); }
#pragma unroll
                for (int qy = 0; qy < M; ++qy) {
                    const T a0 = A0[qy * M], a1 = A1[qy * M], a2 = A2[qy * M];
#pragma unroll
                    for (int by = 0; by < N; ++by) {
                        c0[by] += Bt[qy * N + by] * a0;
                        c12[by] += Dt[qy * N + by] * a1 + Bt[qy * N + by] * a2;
                    }
                }
#pragma unroll
                for (int by = 0; by < N; ++by) {
                    A0[by * M] = c0[by];
                    A0[QS + by * M] = c12[by];
                }
            }
            __syncthreads();
            // x contraction into the (FP64) residual: res = Dx^T C0 + Bx^T C12
            for (int i = tid; i < E * 5 * N2; i += NT) {
                const int e = i / (5 * N2);
                int v, byz;
                task2<TO::xc, 5, N2>(i - e * 5 * N2, v, byz);
                const T* C0 = Q + e * W + (v * 3) * QS + (byz / N) * NF + (byz % N) * M;
                const T* C12 = C0 + QS;
                T r[N];
#pragma unroll
                for (int bx = 0; bx < N; ++bx) r[bx] = T(0);
#pragma unroll
                for (int qx = 0; qx < M; ++qx) {
                    const T c0 = C0[qx], c12 = C12[qx];
#pragma unroll
                    for (int bx = 0; bx < N; ++bx) r[bx] += Dt[qx * N + bx] * c0 + Bt[qx * N + bx] * c12;
                }
                double* res = sRes + e * ES + v * VS;
#pragma unroll
                for (int bx = 0; bx < N; ++bx) res[L::cw(bx, byz % N, byz / N)] = double(r[bx]);
            }
            // with FX the face fluxes must have landed before the lift: their copies
            // are waited for here, so this barrier serves both
            if constexpr (L::FX) cp_async_wait_older();
            __syncthreads();
        } else {
            // ---- fused: z interpolation, Euler flux, contravariant transform and
            //      first (z) divergence contraction; then y and x contractions ----
            T* Abuf = sW + 5 * X2S;                     // [GA][3][X2S] over X1
            T* Cbuf = Abuf + L::GA * 3 * X2S;           // [GA][2][X1S]
            // one (x,y) pencil of element e for variable group g; the buffers hold
            // the group's variables from slot abase (0, or its first variable with PZ)
            auto pencil = [&](auto gc, int e, int qxy) {
                constexpr int g = decltype(gc)::value;
                constexpr int gv0 = group_first<P, G>(g), gnv = group_size<P, G>(g), abase = PZ ? gv0 : 0;
                const int qx = qxy % M, qy = qxy / M;
                T xz[5][N];
#pragma unroll
                for (int v = 0; v < 5; ++v)
#pragma unroll
                    for (int bz = 0; bz < N; ++bz) xz[v][bz] = X2[e * W + v * X2S + bz * NF + qxy];
                const GeoDev* geo = a.geo + sCls[e];
                const T hr = kShift ? T(a.gamma * geo->eref) : T(0);
                const T pref = kShift ? T((a.gamma - 1.0) * geo->eref) : T(0);
                T JD[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) JD[k] = T(geo->JD[k]);
                T acc[gnv][3][N];
#pragma unroll
                for (int v = 0; v < gnv; ++v)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
#pragma unroll
                        for (int bz = 0; bz < N; ++bz) acc[v][d][bz] = T(0);
                const T wxy = Wt[qx] * Wt[qy];
#pragma unroll
                for (int qz = 0; qz < M; ++qz) {
                    T U[5];
#pragma unroll
                    for (int v = 0; v < 5; ++v) {
                        T s = T(0);
#pragma unroll
                        for (int bz = 0; bz < N; ++bz) s += Bt[qz * N + bz] * xz[v][bz];
                        U[v] = s;
                    }
                    T F[15];
                    const T p = dgp::interior_flux_r1<T, kShift>(gamma, U, F, hr);
                    if constexpr (g == 0) {
                        if (!(U[0] > T(0))) status |= kStatusRho;
                        if (!(p + pref > T(0))) status |= kStatusPressure;
                        if (U[0] != U[0] || p != p) status |= kStatusNaN;
                    }
                    const T wq = wxy * Wt[qz];
#pragma unroll
                    for (int vv = 0; vv < gnv; ++vv) {
                        const int v = gv0 + vv;
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const T Gd = (F[v] * JD[d * 3 + 0] + F[5 + v] * JD[d * 3 + 1] + F[10 + v] * JD[d * 3 + 2]) * wq;
#pragma unroll
                            for (int bz = 0; bz < N; ++bz) acc[vv][d][bz] += (d == 2 ? Dt[qz * N + bz] : Bt[qz * N + bz]) * Gd;
                        }
                    }
                }
#pragma unroll
                for (int vv = 0; vv < gnv; ++vv)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
#pragma unroll
                        for (int bz = 0; bz < N; ++bz)
                            Abuf[e * W + ((abase + vv) * 3 + d) * X2S + bz * NF + qxy] = acc[vv][d][bz];
            };
            // y and x contractions of nv buffered variables into residual variables
            // v0 .. v0+nv-1: C0 = By^T A0, C12 = Dy^T A1 + By^T A2; res = Dx^T C0 + Bx^T C12
            auto contract_yx = [&](int nv, int v0) {
                for (int i = tid; i < E * nv * N * M; i += NT) {
                    const int qx = i % M, bz = (i / M) % N, vv = (i / (M * N)) % nv, e = i / (nv * N * M);
                    const T* A0 = Abuf + e * W + (vv * 3 + 0) * X2S + bz * NF + qx;
                    const T* A1 = A0 + X2S;
                    const T* A2 = A1 + X2S;
                    T c0[N], c12[N];
#pragma unroll
                    for (int by = 0; by < N; ++by) { c0[by] = T(0); c12[by] = T(0); }
#pragma unroll
                    for (int qy = 0; qy < M; ++qy) {
                        const T a0 = A0[qy * M], a1 = A1[qy * M], a2 = A2[qy * M];
#pragma unroll
                        for (int by = 0; by < N; ++by) {
                            c0[by] += Bt[qy * N + by] * a0;
                            c12[by] += Dt[qy * N + by] * a1 + Bt[qy * N + by] * a2;
                        }
                    }
                    T* C0 = Cbuf + e * W + (vv * 2) * X1S + bz * N * M + qx;
#pragma unroll
                    for (int by = 0; by < N; ++by) {
                        C0[by * M] = c0[by];
                        C0[X1S + by * M] = c12[by];
                    }
                }
                __syncthreads();
                for (int i = tid; i < E * nv * N2; i += NT) {
                    const int vv = i % nv, byz = (i / nv) % N2, e = i / (nv * N2);
                    const T* C0 = Cbuf + e * W + (vv * 2) * X1S + byz * M;
                    const T* C12 = C0 + X1S;
                    T r[N];
#pragma unroll
                    for (int bx = 0; bx < N; ++bx) r[bx] = T(0);
#pragma unroll
                    for (int qx = 0; qx < M; ++qx) {
                        const T c0 = C0[qx], c12 = C12[qx];
#pragma unroll
                        for (int bx = 0; bx < N; ++bx) r[bx] += Dt[qx * N + bx] * c0 + Bt[qx * N + bx] * c12;
                    }
                    double* res = sRes + e * ES + (v0 + vv) * VS;
#pragma unroll
                    for (int bx = 0; bx < N; ++bx) res[L::cw(bx, byz % N, byz / N)] = double(r[bx]);
                }
                __syncthreads();
            };
            if constexpr (PZ) {
                // every group's pencils in one phase, then all five variables at once
                for (int i = tid; i < E * NF * G; i += NT) {
                    const int g = i / (E * NF), r = i - g * (E * NF);
                    static_for<0, G>([&](auto gc) {
                        if (g == decltype(gc)::value) pencil(gc, r / NF, r % NF);
                    });
                }
                __syncthreads();
                contract_yx(5, 0);
            } else {
                static_for<0, G>([&](auto gc) {
                    for (int i = tid; i < E * NF; i += NT) pencil(gc, i / NF, i % NF);
                    __syncthreads();
                    contract_yx(group_size<P, G>(decltype(gc)::value), group_first<P, G>(decltype(gc)::value));
                });
            }
        }

        if constexpr (!L::FX) {
            // ---- faces: the neighbours' slices have landed (the next batch's
            //      coefficients may still be in flight) ----
            if constexpr (SB) cp_async_wait_all();  // only the slices are in flight
            else cp_async_wait_older();
            __syncthreads();
            // own and neighbour traces: one task per (element, face, variable) doing
            // both sides, or -- when the CTA has threads to spare (high orders) --
            // one task per side
            constexpr bool kSplitSides = 2 * E * 30 <= NT;
            if constexpr (L::RS) {
                // one task per (element, side, face, variable, output row t1):
                // r = sum_b1 B[t1][b1] s[b1][.], then row t1 = sum_b0 B[t0][b0] r[b0]
                for (int t = tid; t < E * 60 * M; t += NT) {
                    const int t1 = t % M, r0 = t / M;
                    const int v = r0 % 5, f = (r0 / 5) % 6, side = (r0 / 30) % 2, e = r0 / 60;
                    // both sides in the own element's energy frame
                    const double sh = kShift && v == 4 ? a.geo[sRec[e * 6].cls].eref : 0.0;
                    // slice entry (b0, b1) at src[b0 * s0 + b1 * s1]
                    // (own side: coefficient index o0 + b0 * s0 + b1 * s1 in the block's layout)
                    const double* src;
                    int s0 = 1, s1 = N, o0 = 0;
                    if (side == 0) {
                        const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
                        src = sU + e * ES + v * VS;
                        o0 = ax == 0 ? sidx : (ax == 1 ? sidx * N : sidx * N2);
                        s0 = ax == 0 ? N : 1;
                        s1 = ax == 2 ? N : N2;
                    } else {
                        src = sOps + e * OPS + (f * 5 + v) * NS;
                    }
                    T r[N];
#pragma unroll
                    for (int b0 = 0; b0 < N; ++b0) r[b0] = T(0);
#pragma unroll
                    for (int b1 = 0; b1 < N; ++b1) {
                        const T c = Bt[t1 * N + b1];
#pragma unroll
                        for (int b0 = 0; b0 < N; ++b0) {
                            const int k = o0 + b0 * s0 + b1 * s1;
                            const double x = src[side == 0 ? L::cwl(k) : k];
                            r[b0] += c * (kShift ? T(x - sh) : T(x));
                        }
                    }
                    T* o = sW + e * W + side * 30 * FS + (f * 5 + v) * FS + t1 * M;
#pragma unroll
                    for (int t0 = 0; t0 < M; ++t0) {
                        T sum = T(0);
#pragma unroll
                        for (int b0 = 0; b0 < N; ++b0) sum += Bt[t0 * N + b0] * r[b0];
                        o[t0] = sum;
                    }
                }
            } else if constexpr (kSplitSides) {
                for (int t = tid; t < E * 60; t += NT) {
                    const int v = t % 5, f = (t / 5) % 6, side = (t / 30) % 2, e = t / 60;
                    // both sides in the own element's energy frame
                    const double sh = kShift && v == 4 ? a.geo[sRec[e * 6].cls].eref : 0.0;
                    T sl[N][N];
                    if (side == 0) {
                        const double* own = sU + e * ES + v * VS;
#pragma unroll
                        for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                            for (int b0 = 0; b0 < N; ++b0)
                                sl[b1][b0] =
                                    kShift ? T(own[L::cwl(slice_index<N>(f, b0, b1))] - sh) : T(own[L::cwl(slice_index<N>(f, b0, b1))]);
                    } else {
                        const double* nb = sOps + e * OPS + (f * 5 + v) * NS;
#pragma unroll
                        for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                            for (int b0 = 0; b0 < N; ++b0)
                                sl[b1][b0] = kShift ? T(nb[b1 * N + b0] - sh) : T(nb[b1 * N + b0]);
                    }
                    interp2d<N, M, T>(Bt, sl, sW + e * W + side * 30 * FS + (f * 5 + v) * FS);
                }
            } else {
                for (int t = tid; t < E * 30; t += NT) {
                    const int v = t % 5, f = (t / 5) % 6, e = t / 30;
                    T sn[N][N], so[N][N];
                    const double* nb = sOps + e * OPS + (f * 5 + v) * NS;
                    const double* own = sU + e * ES + v * VS;
                    // both sides in the own element's energy frame
                    const double sh = kShift && v == 4 ? a.geo[sRec[e * 6].cls].eref : 0.0;
#pragma unroll
                    for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                        for (int b0 = 0; b0 < N; ++b0) {
                            sn[b1][b0] = kShift ? T(nb[b1 * N + b0] - sh) : T(nb[b1 * N + b0]);
                            so[b1][b0] = kShift ? T(own[L::cwl(slice_index<N>(f, b0, b1))] - sh) : T(own[L::cwl(slice_index<N>(f, b0, b1))]);
                        }
                    interp2d<N, M, T>(Bt, so, sW + e * W + (f * 5 + v) * FS);
                    interp2d<N, M, T>(Bt, sn, sW + e * W + 30 * FS + (f * 5 + v) * FS);
                }
            }
            __syncthreads();
            // the staging area is free: stream in this batch's RK operands (and,
            // with SB, the next batch's coefficients: the traces were their last reader)
            if (stage_u0) prefetch_batch<P, G, E, NT>(a.U0, a.ne, e0, sOps, OPS);
            if (need_u0_acc) prefetch_batch<P, G, E, NT>(a.acc, a.ne, e0, sOps + ES, OPS);
            if (SB && en < a.ne) prefetch_batch<P, G, E, NT>(a.Us, a.ne, en, sU, ES);
            cp_async_commit();

            // numerical flux at every face point, written over the own trace; two
            // points per thread and iteration for instruction-level parallelism
            {
                constexpr int total = E * 6 * NF;
                auto point = [&](int i, T (&Fo)[5], int& off) {
                    const int cidx = i % NF, f = (i / NF) % 6, e = i / (6 * NF);
                    const int fm = e * 6 + f;
                    const FaceRec& rec = sRec[fm];
                    const int isL = (rec.info >> 3) & 1;
                    const int cn = sCm[fm * NF + cidx];
                    const T* Tr = sW + e * W + f * 5 * FS;
                    const T* Tn = sW + e * W + 30 * FS + f * 5 * FS;
                    T UL[5], UR[5];
#pragma unroll
                    for (int v = 0; v < 5; ++v) {
                        const T uo = Tr[v * FS + cidx], un = Tn[v * FS + cn];
                        UL[v] = isL ? uo : un;  // element-wise selects keep both in registers
                        UR[v] = isL ? un : uo;
                    }
                    // the left element's normal data: per face, or per face point (GE)
                    T nd[4];
                    if constexpr (L::GE) {
                        const double* gn = a.gnrm + ((size_t)min(e0 + e, a.ne - 1) * 6 + f) * 4 * NF + cidx;
#pragma unroll
                        for (int k = 0; k < 4; ++k) nd[k] = T(gn[k * NF]);
                    } else {
                        nd[0] = T(rec.n[0]);
                        nd[1] = T(rec.n[1]);
                        nd[2] = T(rec.n[2]);
                        nd[3] = T(rec.nmag);
                    }
                    const double eref = kShift ? a.geo[sRec[e * 6].cls].eref : 0.0;
                    numerical_flux<T, kShift>(a.flux, a.gamma, UL, UR, nd, eref, Fo, status);
                    const T w = Wt[cidx % M] * Wt[cidx / M];
                    const T sgn = isL ? T(-1.0) : T(1.0);
#pragma unroll
                    for (int v = 0; v < 5; ++v) Fo[v] = sgn * (Fo[v] * w);
                    off = e * W + f * 5 * FS + cidx;
                };
                // KP independent points per thread and iteration (latency hiding)
                constexpr int KP = kFluxPoints;
                for (int i0 = tid; i0 < total; i0 += KP * NT) {
                    T Fk[KP][5];
                    int ok[KP];
#pragma unroll
                    for (int k = 0; k < KP; ++k) {
                        const int ik = i0 + k * NT;
                        point(ik < total ? ik : i0, Fk[k], ok[k]);
                    }
#pragma unroll
                    for (int k = 0; k < KP; ++k)
                        if (k == 0 || i0 + k * NT < total) {
#pragma unroll
                            for (int v = 0; v < 5; ++v) sW[ok[k] + v * FS] = Fk[k][v];
                        }
                }
            }
            __syncthreads();

            // the face records have been read: queue the next batch's (they land
            // before the inverse-mass pass, which waits for all copies)
            if (en < a.ne) prefetch_recs<E, NT>(a.frec, a.ne, en, sRec);
            cp_async_commit();
        } else if constexpr (!L::UF) {
            // the face fluxes have landed (the next batch's coefficients may
            // still be in flight; the unfused volume waited for them before
            // its last barrier)
            cp_async_wait_older();
            __syncthreads();
        }
        // face lift per (element, face, variable) into Tn's space
        // the face flux of (element e, face f): in the trace area, or with FX the
        // face kernel's flux staged in the operand region, negated for the left side
        auto face_flux_in = [&](int e, int f) -> const T* {
            if constexpr (L::FX) return reinterpret_cast<const T*>(sOps + e * OPS) + f * 5 * FS;
            else return sW + e * W + f * 5 * FS;
        };
        auto face_sign = [&](int e, int f) -> T {
            if constexpr (L::FX) return ((sRec[e * 6 + f].info >> 3) & 1) ? T(-1.0) : T(1.0);
            else return T(1.0);
        };
        if constexpr (L::RS) {
            // one task per (element, face, variable, output row b1)
            for (int t = tid; t < E * 30 * N; t += NT) {
                const int b1 = t % N, r0 = t / N;
                const int v = r0 % 5, f = (r0 / 5) % 6, e = r0 / 30;
                const T* Fq = face_flux_in(e, f) + v * FS;
                const T sgn = face_sign(e, f);
                T r[M];
#pragma unroll
                for (int t0 = 0; t0 < M; ++t0) r[t0] = T(0);
#pragma unroll
                for (int t1 = 0; t1 < M; ++t1) {
                    const T c = Bt[t1 * N + b1];
#pragma unroll
                    for (int t0 = 0; t0 < M; ++t0) r[t0] += c * Fq[t1 * M + t0];
                }
                T* Lf = sW + e * W + 30 * FS + (f * 5 + v) * FS + b1 * N;
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) {
                    T sum = T(0);
#pragma unroll
                    for (int t0 = 0; t0 < M; ++t0) sum += Bt[t0 * N + b0] * r[t0];
                    Lf[b0] = L::FX ? sgn * sum : sum;
                }
            }
        } else {
            for (int t = tid; t < E * 30; t += NT) {
                const int v = t % 5, f = (t / 5) % 6, e = t / 30;
                const T* Fq = face_flux_in(e, f) + v * FS;
                const T sgn = face_sign(e, f);
                T tmp[M][N];
#pragma unroll
                for (int t1 = 0; t1 < M; ++t1)
#pragma unroll
                    for (int b0 = 0; b0 < N; ++b0) {
                        T s = T(0);
#pragma unroll
                        for (int t0 = 0; t0 < M; ++t0) s += Bt[t0 * N + b0] * Fq[t1 * M + t0];
                        tmp[t1][b0] = s;
                    }
                T* Lf = sW + e * W + 30 * FS + (f * 5 + v) * FS;
#pragma unroll
                for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                    for (int b0 = 0; b0 < N; ++b0) {
                        T s = T(0);
#pragma unroll
                        for (int t1 = 0; t1 < M; ++t1) s += Bt[t1 * N + b1] * tmp[t1][b0];
                        Lf[b1 * N + b0] = L::FX ? sgn * s : s;
                    }
            }
        }
        __syncthreads();
        if constexpr (L::FX) {
            // the staged fluxes and the face records have been read: stream in this
            // batch's RK operands and the next batch's records
            if (stage_u0) prefetch_batch<P, G, E, NT>(a.U0, a.ne, e0, sOps, OPS);
            if (need_u0_acc) prefetch_batch<P, G, E, NT>(a.acc, a.ne, e0, sOps + ES, OPS);
            if (en < a.ne) prefetch_recs<E, NT>(a.frec, a.ne, en, sRec);
            cp_async_commit();
        }
        // add the six face contributions to the (FP64) residual (with MG, in
        // the inverse mass's x pass, except for the residual output)
        const bool fold_lifts = L::MG && a.mode != kModeResidual;
        for (int i = tid; i < (fold_lifts ? 0 : E * 5 * NB); i += NT) {
            const int e = i / (5 * NB);
            int b, v;
            task2<TO::gather, NB, 5>(i - e * 5 * NB, b, v);
            const int bc[3] = {b % N, (b / N) % N, b / N2};
            const T* Lf = sW + e * W + 30 * FS + v * FS;
            double s = 0.0;
            if constexpr (L::GE && kShift) {
                if (v >= 1 && v <= 3)
                    s = (a.gamma - 1.0) * a.geo[sCls[e]].eref * a.gfsd[(size_t)min(e0 + e, a.ne - 1) * 5 * NB + v * NB + b];
            }
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
                if (bc[ax] == sidx) {
                    const int b0 = ax == 0 ? bc[1] : bc[0];
                    const int b1 = ax == 2 ? bc[1] : bc[2];
                    s += double(Lf[f * 5 * FS + b1 * N + b0]);
                }
            }
            sRes[e * ES + v * VS + L::cw(bc[0], bc[1], bc[2])] += s;
        }
        if (!fold_lifts) __syncthreads();

        if (a.mode == kModeResidual) {
            for (int i = tid; i < E * 5 * NB; i += NT) {
                const int e = i / (5 * NB), r = i - e * (5 * NB), v = r / NB, b = r - v * NB;
                if (e0 + e < a.ne) a.out[(size_t)e0 * 5 * NB + i] = sRes[e * ES + v * VS + L::cwl(b)];
            }
            continue;
        }

        if constexpr (L::GE) {
            // ---- dense inverse mass (FP64, the element's own matrix) fused with
            //      the update: one task per (element, basis function), the five
            //      variables together; the matrix streams from global memory ----
            cp_async_wait_all();  // this batch's U0 / accumulator have landed
            __syncthreads();
            for (int i = tid; i < E * NB; i += NT) {
                const int j = i % NB, e = i / NB;
                if (e0 + e >= a.ne) continue;
                const int ge = e0 + e;
                const double* im = a.gimm + (size_t)ge * NB * NB + j;  // iMM[j][k] at im[k * NB]
                const double* r = sRes + e * ES;
                double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                for (int kz = 0; kz < N; ++kz)
#pragma unroll
                    for (int ky = 0; ky < N; ++ky)
#pragma unroll
                        for (int kx = 0; kx < N; ++kx) {
                            const double mk = im[(size_t)((kz * N + ky) * N + kx) * NB];
                            const int kw = L::cw(kx, ky, kz);
#pragma unroll
                            for (int v = 0; v < 5; ++v) s[v] += mk * r[v * VS + kw];
                        }
                const double scale = a.dt * a.geo[sCls[e]].dtf;
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    const double kk = scale * s[v];
                    const size_t gi = (size_t)ge * 5 * NB + (size_t)v * NB + j;
                    // step-start state: the prefetched U0, or the stage state itself in RK1 / FE
                    const int jw = L::cwl(j);
                    const double u0 = stage_u0 ? sOps[e * OPS + v * VS + jw] : sU[e * ES + v * VS + jw];
                    const double ac = sOps[e * OPS + ES + v * VS + jw];
                    switch (a.mode) {
                        case kModeMassInv: a.out[gi] = kk; break;
                        case kModeRK1: a.acc[gi] = kk; a.out[gi] = 0.5 * kk + u0; break;
                        case kModeRK2: a.acc[gi] = ac + 2.0 * kk; a.out[gi] = 0.5 * kk + u0; break;
                        case kModeRK3: a.acc[gi] = ac + 2.0 * kk; a.out[gi] = 1.0 * kk + u0; break;
                        case kModeRK4: a.out[gi] = u0 + (1.0 / 6.0) * (ac + kk); break;
                        default: a.out[gi] = u0 + 1.0 * kk; break;
                    }
                }
            }
        } else {
            // ---- inverse mass (FP64): x and y passes in place, z pass fused with the update ----
            for (int i = tid; i < E * 5 * N2; i += NT) {
                const int e = i / (5 * N2);
                int v, byz;
                task2<(L::MG ? TO::minvxg : TO::minvx), 5, N2>(i - e * 5 * N2, v, byz);
                const int by = byz % N, bz = byz / N;
                double* r = sRes + e * ES + v * VS;  // pencil along x
                double t[N];
#pragma unroll
                for (int k = 0; k < N; ++k) t[k] = r[L::cw(k, by, bz)];
                if constexpr (L::MG) {
                    // the face contributions of the pencil's coefficients, summed
                    // in face order and added as the separate pass adds them
                    const T* Lf = sW + e * W + 30 * FS + v * FS;
#pragma unroll
                    for (int k = 0; k < N; ++k) {
                        const int bc[3] = {k, by, bz};
                        double s = 0.0;
#pragma unroll
                        for (int f = 0; f < 6; ++f) {
                            const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
                            if (bc[ax] == sidx) {
                                const int b0 = ax == 0 ? bc[1] : bc[0];
                                const int b1 = ax == 2 ? bc[1] : bc[2];
                                s += double(Lf[f * 5 * FS + b1 * N + b0]);
                            }
                        }
                        t[k] += s;
                    }
                }
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    double s = 0.0;
#pragma unroll
                    for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t[k];
                    r[L::cw(j, by, bz)] = s;
                }
            }
            __syncthreads();
            for (int i = tid; i < E * 5 * N2; i += NT) {
                const int e = i / (5 * N2);
                int v, bx, bz;
                task3<TO::minvy, 5, N, N>(i - e * 5 * N2, v, bx, bz);
                double* r = sRes + e * ES + v * VS;  // pencil along y
                double t[N];
#pragma unroll
                for (int k = 0; k < N; ++k) t[k] = r[L::cw(bx, k, bz)];
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    double s = 0.0;
#pragma unroll
                    for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t[k];
                    r[L::cw(bx, j, bz)] = s;
                }
            }
            cp_async_wait_all();  // this batch's U0 / accumulator have landed
            __syncthreads();
            for (int i = tid; i < E * 5 * N2; i += NT) {
                const int bxy = i % N2, ev = i / N2, e = ev / 5;
                if (e0 + e >= a.ne) continue;
                const int ge = e0 + e;
                const GeoDev& gg = a.geo[sCls[e]];
                const double scale = a.dt * gg.dtf * gg.inv_djac;
                const int v = ev % 5;
                // pencil along z: (bx, by, k) at word L::cw(bx, by, k) of each block
                const int bx = bxy % N, by = bxy / N;
                const double* r = sRes + e * ES + v * VS;
                // step-start state: the prefetched U0, or the stage state itself in
                // RK1 / FE where the two coincide
                const double* u0 = (stage_u0 ? sOps + e * OPS : sU + e * ES) + v * VS;
                const double* ac = sOps + e * OPS + ES + v * VS;
                double t[N];
#pragma unroll
                for (int k = 0; k < N; ++k) t[k] = r[L::cw(bx, by, k)];
                const size_t gbase = (size_t)e0 * 5 * NB + (size_t)ev * NB + bxy;
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    double s = 0.0;
#pragma unroll
                    for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t[k];
                    const double kk = scale * s;
                    const size_t gi = gbase + (size_t)j * N2;
                    const int jw = L::cw(bx, by, j);
                    switch (a.mode) {
                        case kModeMassInv: a.out[gi] = kk; break;
                        case kModeRK1: a.acc[gi] = kk; a.out[gi] = 0.5 * kk + u0[jw]; break;
                        case kModeRK2: a.acc[gi] = ac[jw] + 2.0 * kk; a.out[gi] = 0.5 * kk + u0[jw]; break;
                        case kModeRK3: a.acc[gi] = ac[jw] + 2.0 * kk; a.out[gi] = 1.0 * kk + u0[jw]; break;
                        case kModeRK4: a.out[gi] = u0[jw] + (1.0 / 6.0) * (ac[jw] + kk); break;
                        default: a.out[gi] = u0[jw] + 1.0 * kk; break;
                    }
                }
            }
        }
    }
    cp_async_wait_all();
    if (status) atomicOr(a.status, status);
}

// ---- launch option FX: the face kernel ----
// Every interior face's numerical flux, once: per batch of FB faces, both
// sides' boundary slices (gathered from the state into registers, one task per
// face side and variable), their traces (2D interpolation), and at
// each point of the listed side's face grid (the left side, or an owned right
// side facing a ghost) the flux in the reference's L/R convention with the
// left element's normal (both states in the listed side's energy frame),
// times the point's quadrature weight, written to fflux[face][5][(p+2)^2] in
// the listed side's canonical point order.  The same operations as the stage kernel's own face
// phase (flux_functors_impl.h:168-264), done once per face instead of once per
// side.
// faces per batch (measured best: 12 for the FP64 kernel at every order, one
// round of 120 gather tasks on 128 threads; for the FP32 one 16 up to p = 3
// and 8 above) and threads of the face kernel
__host__ __device__ constexpr int face_batch_of(int p, int bytes) { return bytes == 8 ? 12 : (p <= 3 ? 16 : 8); }
template <int P, typename T>
__host__ __device__ constexpr int face_batch() { return face_batch_of(P, sizeof(T)); }
constexpr int kFaceThreads = 128;
// threads of the standalone face kernel: one round of the batch's gather tasks
// (faces x 2 sides x 5 variables), at least 128
template <int P, typename T>
__host__ __device__ constexpr int face_threads()
{
    return (face_batch<P, T>() * 10 + 31) / 32 * 32 > kFaceThreads ? (face_batch<P, T>() * 10 + 31) / 32 * 32
                                                                    : kFaceThreads;
}

template <int P, typename T>
constexpr size_t face_smem_bytes()
{
    using L = Lay<P, 1, T>;
    constexpr int FB = face_batch<P, T>();
    // traces, then two buffers of the batch's face records (the next batch's are
    // fetched while this one computes) and listed elements / faces
    return ((sizeof(T) * FB * 10 * L::FS + 15) / 16) * 16 + 2 * FB * sizeof(FaceRec) + 4 * FB * sizeof(int);
}

// GEO: general geometry, the left element's normal data per face point;
// bid / nblk as for stage_body
template <int P, typename T, bool GEO, int NTF = kFaceThreads>
__device__ __forceinline__ void face_flux_body(const StageArgs& a, int bid, int nblk, int* work = nullptr,
                                               int* slots = nullptr)
{
    using L = Lay<P, 1, T>;
    constexpr int FB = face_batch<P, T>(), NT = NTF;
    constexpr int N = L::N, M = L::M, NB = L::NB, NF = L::NF, N2 = L::N2, FS = L::FS;
    constexpr bool kShift = sizeof(T) == 4;
    extern __shared__ double fsm[];
    T* sTr = reinterpret_cast<T*>(fsm);                                             // [FB][2][5][FS]
    unsigned char* tail = reinterpret_cast<unsigned char*>(sTr) + ((sizeof(T) * FB * 10 * FS + 15) / 16) * 16;
    FaceRec* sRecBuf = reinterpret_cast<FaceRec*>(tail);                            // [2][FB] listed side's records
    int* sELBuf = reinterpret_cast<int*>(sRecBuf + 2 * FB);                         // [2][FB] listed elements
    int* sFLBuf = sELBuf + 2 * FB;                                                  // [2][FB] listed faces
    const T* __restrict__ Bt = TabSel<T>::B(a.tab);
    const T* __restrict__ Wt = TabSel<T>::W(a.tab);
    T* out = reinterpret_cast<T*>(a.fflux);
    const int tid = threadIdx.x;
    unsigned status = 0;
    // batches of faces: static (bid, nblk) or claimed one ahead (work, slots), as in stage_body
    int f_first = a.face_begin + bid * FB;
    if (work) {
        if (tid == 0) {
            slots[0] = a.face_begin + atomicAdd(work, 1) * FB;
            slots[1] = a.face_begin + atomicAdd(work, 1) * FB;
        }
        __syncthreads();
        f_first = slots[0];
    }
    // the records of batch f into buffer rb: listed (element, face), then the
    // listed side's face record by cp.async (waited for at the next batch's top)
    auto fetch_records = [&](int f, int rb, int2 fe) {
        if (tid < FB && f < a.nface) {
            sELBuf[rb * FB + tid] = fe.x;
            sFLBuf[rb * FB + tid] = fe.y;
            const double* src = reinterpret_cast<const double*>(a.frec + (size_t)fe.x * 6 + fe.y);
            double* dst = reinterpret_cast<double*>(sRecBuf + rb * FB + tid);
#pragma unroll
            for (int w = 0; w < 6; ++w) cp_async8(dst + w, src + w);
        }
        cp_async_commit();
    };
    int fn = f_first, it = 0;
    if (f_first < a.nface)
        fetch_records(f_first, 0, tid < FB ? a.faces[min(f_first + tid, a.nface - 1)] : make_int2(0, 0));
    for (int f0 = f_first; f0 < a.nface; f0 = fn, ++it) {
        const int rb = it & 1;
        FaceRec* sRecL = sRecBuf + rb * FB;
        const int* sEL = sELBuf + rb * FB;
        const int* sFL = sFLBuf + rb * FB;
        cp_async_wait_all();
        __syncthreads();
        if (work) {
            fn = slots[(it + 1) & 1];
            if (tid == 0) slots[it & 1] = a.face_begin + atomicAdd(work, 1) * FB;
        } else {
            fn = f0 + nblk * FB;
        }
        // the next batch's face list entries, in flight during the traces
        const int2 fe_next = tid < FB && fn < a.nface ? a.faces[min(fn + tid, a.nface - 1)] : make_int2(0, 0);
        // traces of both sides, in the left element's energy frame: one task per
        // (face, side, variable) gathers its boundary slice from the state into
        // registers (entry (b0, b1) at coefficient o0 + b0 s0 + b1 s1)
        for (int t = tid; t < FB * 10; t += NT) {
            const int v = t % 5, sj = t / 5, j = sj / 2, side = sj % 2;
            const FaceRec& rec = sRecL[j];
            const int el = side == 0 ? sEL[j] : rec.nbr;
            const int fc = side == 0 ? sFL[j] : (rec.info & 7);
            const int ax = face_axis(fc), sidx = face_side(fc) ? N - 1 : 0;
            const int o0 = ax == 0 ? sidx : (ax == 1 ? sidx * N : sidx * N2);
            const int s0 = ax == 0 ? N : 1, s1 = ax == 2 ? N : N2;
            const double* src = a.Us + ((size_t)el * 5 + v) * NB + o0;
            const double sh = kShift && v == 4 ? a.geo[rec.cls].eref : 0.0;
            double x[N][N];
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) x[b1][b0] = __ldg(src + b0 * s0 + b1 * s1);
            T sl[N][N];
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) sl[b1][b0] = kShift ? T(x[b1][b0] - sh) : T(x[b1][b0]);
            interp2d<N, M, T>(Bt, sl, sTr + (sj * 5 + v) * FS);
        }
        // the next batch's records stream in while this batch's fluxes compute
        fetch_records(fn, rb ^ 1, fe_next);
        __syncthreads();
        // the flux at the listed side's face points
        for (int i = tid; i < FB * NF; i += NT) {
            const int c = i % NF, j = i / NF;
            if (f0 + j >= a.nface) continue;
            const FaceRec& rec = sRecL[j];
            const int cn = a.cmap[(rec.info >> 4) * NF + c];
            const int isL = (rec.info >> 3) & 1;
            const T* To = sTr + (j * 2) * 5 * FS;  // the listed side
            const T* Tn = To + 5 * FS;             // the other side
            T UL[5], UR[5], Fo[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const T uo = To[v * FS + c], un = Tn[v * FS + cn];
                UL[v] = isL ? uo : un;
                UR[v] = isL ? un : uo;
            }
            T nd[4];
            if constexpr (GEO) {
                const double* gn = a.gnrm + ((size_t)sEL[j] * 6 + sFL[j]) * 4 * NF + c;
#pragma unroll
                for (int k = 0; k < 4; ++k) nd[k] = T(gn[k * NF]);
            } else {
                nd[0] = T(rec.n[0]);
                nd[1] = T(rec.n[1]);
                nd[2] = T(rec.n[2]);
                nd[3] = T(rec.nmag);
            }
            const double eref = kShift ? a.geo[rec.cls].eref : 0.0;
            numerical_flux<T, kShift>(a.flux, a.gamma, UL, UR, nd, eref, Fo, status);
            const T w = Wt[c % M] * Wt[c / M];
            T* o = out + (size_t)(f0 + j) * a.fstride + c;
#pragma unroll
            for (int v = 0; v < 5; ++v) o[v * NF] = Fo[v] * w;
        }
    }
    cp_async_wait_all();
    if (status) atomicOr(a.status, status);
}

template <int P, typename T, bool GEO>
__global__ void __launch_bounds__(face_threads<P, T>()) face_flux_kernel(StageArgs a)
{
    face_flux_body<P, T, GEO, face_threads<P, T>()>(a, blockIdx.x, gridDim.x);
}

template <int P, int E, int NT, int G, typename T, int FL>
__global__ void __launch_bounds__(NT) stage_kernel(StageArgs a)
{
    stage_body<P, E, NT, G, T, FL>(a, blockIdx.x, gridDim.x);
}
// the same with at least MB resident CTAs per SM asked of the compiler (it then
// keeps the registers within 64K / (NT * MB) per thread)
template <int P, int E, int NT, int G, typename T, int FL, int MB>
__global__ void __launch_bounds__(NT, MB) stage_kernel_mb(StageArgs a)
{
    stage_body<P, E, NT, G, T, FL>(a, blockIdx.x, gridDim.x);
}

template <int P, int E, int G, typename T, int FL = 0>
constexpr size_t stage_smem_bytes()
{
    using L = Lay<P, G, T, FL>;
    return ((E * L::bytes_per_elem + 15) / 16) * 16 + E * L::meta_bytes_per_elem;
}

// ---- compiled launch variants (one translation unit per order) ----

struct StageVariant {
    int E, NT, G;        // elements per CTA, threads per CTA, variable groups
    int fp32;            // 1: residual arithmetic in FP32 (mixed precision), 0: FP64
    int flags;           // 1: groups' pencils in one phase, 2: single coefficient buffer,
                         // 4: unfused volume, 8: row-split traces and lifts,
                         // 16: one face-flux point per thread, 32: general (trilinear) geometry,
                         // 64: face fluxes from the face kernel, 128: the tensor-core kernel;
                         // bits 8..11: minimum resident CTAs asked of the compiler (0: none)
    size_t smem;         // dynamic shared memory per CTA
    const void* func;    // the kernel, for attributes / occupancy queries
    cudaError_t (*launch)(const StageArgs&, int grid, cudaStream_t);
    // FX variants: the face kernel launched before the stage kernel (else null)
    const void* face_func;
    size_t face_smem;
    int face_threads;
    cudaError_t (*face_launch)(const StageArgs&, int grid, cudaStream_t);
    int face_batch;      // faces per CTA batch of the face kernel
};

template <int P, typename T, bool GEO>
cudaError_t launch_face_kernel(const StageArgs& a, int grid, cudaStream_t s)
{
    face_flux_kernel<P, T, GEO><<<grid, face_threads<P, T>(), face_smem_bytes<P, T>(), s>>>(a);
    return cudaGetLastError();
}

template <int P, int E, int NT, int G, typename T, int FL, int MB>
cudaError_t launch_stage_variant(const StageArgs& a, int grid, cudaStream_t s)
{
    if constexpr (MB > 0)
        stage_kernel_mb<P, E, NT, G, T, FL, MB><<<grid, NT, stage_smem_bytes<P, E, G, T, FL>(), s>>>(a);
    else
        stage_kernel<P, E, NT, G, T, FL><<<grid, NT, stage_smem_bytes<P, E, G, T, FL>(), s>>>(a);
    return cudaGetLastError();
}

// launch options FL (see Lay); one-phase groups pay off when E * (p+2)^2 * G
// pencil tasks fill fewer rounds of NT threads than G sequential phases; the
// single buffer trades prefetch overlap for occupancy; the unfused volume, the
// row-split traces and the single flux point trade shared-memory traffic for
// parallel tasks and registers (high orders); general geometry is a property
// of the mesh, not a tuning choice: contexts on non-affine meshes run GE
// variants only, the others never do
constexpr int kPZ = 1, kSB = 2, kUF = 4, kRS = 8, kK1 = 16, kGE = 32, kFX = 64, kMG = 4096;
// the tensor-core stage kernel (dg_tc.cuh): a kernel of its own, not an option of stage_kernel
constexpr int kTC = 128;
// MB > 0: at least MB resident CTAs per SM asked of the compiler (a register cap)
template <int P, int E, int NT, int G, typename T = double, int FL = 0, int MB = 0>
StageVariant make_variant()
{
    static_assert(stage_smem_bytes<P, E, G, T, FL>() <= 227 * 1024, "stage kernel shared memory exceeds 227 KB");
    static_assert(MB >= 0 && MB < 16, "minimum resident CTAs out of range");
    const void* func;
    if constexpr (MB > 0) func = (const void*)stage_kernel_mb<P, E, NT, G, T, FL, MB>;
    else func = (const void*)stage_kernel<P, E, NT, G, T, FL>;
    StageVariant v{E, NT, G, sizeof(T) == 4 ? 1 : 0, FL | (MB << 8), stage_smem_bytes<P, E, G, T, FL>(),
                   func, launch_stage_variant<P, E, NT, G, T, FL, MB>, nullptr, 0, 0, nullptr, 0};
    if constexpr ((FL & 64) != 0) {
        static_assert(face_smem_bytes<P, T>() <= 227 * 1024, "face kernel shared memory exceeds 227 KB");
        constexpr bool geo = (FL & 32) != 0;
        v.face_func = (const void*)face_flux_kernel<P, T, geo>;
        v.face_smem = face_smem_bytes<P, T>();
        v.face_threads = face_threads<P, T>();
        v.face_launch = launch_face_kernel<P, T, geo>;
        v.face_batch = face_batch<P, T>();
    }
    return v;
}

// the variants compiled for order p (defined in dg_stage_p<p>.cu)
int stage_variants(int p, const StageVariant** out);
// the tensor-core kernel's operator table of order p from the 1D basis
// B1[q * (p+1) + b] at the GL points, as BF16 bit patterns (false: no
// tensor-core kernel for p), and its face-flux stride (FP32 elements per face)
bool tc_operator(int p, const double* B1, std::vector<uint16_t>& out);
int tc_face_stride(int p);
int stage_variants_p0(const StageVariant** out);
int stage_variants_p1(const StageVariant** out);
int stage_variants_p2(const StageVariant** out);
int stage_variants_p3(const StageVariant** out);
int stage_variants_p4(const StageVariant** out);
int stage_variants_p5(const StageVariant** out);

}  // namespace dgk
