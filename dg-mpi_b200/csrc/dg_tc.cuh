// dg_tc.cuh -- the tensor-core stage kernel (sm_100a, tcgen05): the volume
// integral of the FP32 residual as split-TF32 products on the 5th-generation
// tensor cores, with FP32 accumulation in tensor memory (TMEM).
//
// Reference path replaced (as in dg_stage.cuh): evaluate_state B*U
// (src/solver/helpers.cpp:185-198, Math::cAxB_to_C linear_algebra.cpp:236-241),
// VolumeFluxesFunctor (flux_functors_impl.h:46-115), the grad-basis^T
// contraction calculate_volume_flux_integral (src/solver/tools.cpp:7-35),
// the face lift (tools.cpp:38-63), the inverse mass and the RK stage update
// (stepper.cpp:23-142).  The face fluxes come from face_flux_kernel (launch
// option FX), computed once per face.
//
// Per tile of E elements (one CTA per SM, grid-stride over tiles):
//   GEMM1  D1[q][c] = sum_b B[q][b] U[c][b]      (M = 128 volume points, N = the
//          tile's (element, variable) columns, K = nb): the state at every
//          quadrature point, one TMEM lane per point, so one thread holds all
//          five variables of a point and evaluates the Euler flux in registers;
//   flux   G_d[c][q] = (sum_j F_j(U_q) (ijac djac)[d][j]) w_q, written to shared
//          memory as the A operand of GEMM2 (rows 32 d + c, K = q);
//   GEMM2  H[32 d + c][b] = sum_q G_d[c][q] B[q][b]  (M = 128, N = nb, K = 128):
//          the weak divergence factorised through the basis, D_d = B Delta_d with
//          Delta_d the nodal derivative matrix along axis d (exact: the
//          derivative of a degree-p Lagrange polynomial is interpolated exactly
//          at the p+1 nodes), so res = sum_d Delta_d^T H_d -- one operator, B,
//          serves both GEMMs: K-major as GEMM1's A, MN-major as GEMM2's B;
//   then, on the CUDA cores, Delta_d^T along each axis (FP32), the face lift of
//   the face kernel's fluxes (FP32), the sum into the FP64 residual, the
//   Kronecker inverse mass and the RK stage update in FP64.
// Split products: every operand x is stored as hi = tf32(x), lo = tf32(x - hi)
// and each GEMM accumulates lo*hi + hi*lo + hi*hi (the small terms first).
// The state enters as U - E_ref in its energy (the FP32 residual's energy
// reference, see dgp::interior_flux_r1).
//
// Shared-memory operands use the 128-byte swizzled canonical layout of the
// UMMA descriptors: atoms of 8 rows x 128 bytes (32 four-byte elements along
// the atom's row), 1024-byte aligned, with the 16-byte chunk index of a row
// XORed with the row's index within the atom.  Every wait on an mbarrier is
// bounded (clock64); a wait that gives up sets kStatusTimeout, the CTA stops,
// releases its TMEM and returns.  No multicast, no peer memory: every operand
// is in this CTA's own shared memory.
#pragma once
#include <cstdint>
#include <cstring>

#include "dg_stage.cuh"

namespace dgk {

constexpr unsigned kStatusTimeout = 16u;

namespace tc {

// ---- PTX wrappers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// one poll of the phase with parity `parity`
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// waits until the phase completes or about `limit` SM cycles have passed
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit)
{
    const long long t0 = clock64();
    while (!mbar_test(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
// bulk copy global -> this CTA's shared memory, completing on an mbarrier
// (both addresses 16-byte aligned, bytes a multiple of 16; no multicast)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_slot), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// D (TMEM, FP32) (+)= A (smem) * B (smem), kind::tf32, issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
// arrives on the mbarrier once every MMA issued so far by this thread is complete
__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

// TMEM -> registers: this warp's 32 lanes (lane quarter warp % 4), consecutive columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&r)[8])
{
    uint32_t u[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) r[i] = __uint_as_float(u[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* r)
{
    uint32_t u[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
          "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(u[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// round to TF32 (10 explicit mantissa bits), to nearest, ties away from zero
__device__ __forceinline__ float tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// ---- descriptors ----
// shared-memory matrix descriptor, 128-byte swizzle (layout type 2), version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}
// instruction descriptor of kind::tf32 with FP32 accumulation: M rows, N
// columns, A K-major, B K-major (b_mn = 0) or MN-major (b_mn = 1)
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int b_mn)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(b_mn) << 16) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// byte offset of element (row, k) of a four-byte operand in 128-byte swizzled
// atoms: 8-row groups at 1024 bytes, 32-element atoms along k at `katom` bytes
__host__ __device__ constexpr uint32_t sw128(int row, int k, int katom)
{
    return static_cast<uint32_t>((k >> 5) * katom + (row >> 3) * 1024 + (row & 7) * 128 +
                                 ((((k & 31) >> 2) ^ (row & 7)) << 4) + (k & 3) * 4);
}

}  // namespace tc

// ---- the kernel's configuration per order (p = 3: nb = 64, 125 volume points) ----
template <int P>
struct TcCfg;
template <>
struct TcCfg<3> {
    static constexpr int N = 4, M = 5, NB = 64, NQ = 125, NF = 25, FS = 25;
    static constexpr int E = 6;            // elements per tile
    static constexpr int C = 5 * E;        // (element, variable) columns of a tile (30)
    static constexpr int N1 = 32;          // GEMM1 N: the columns, padded to 32
    static constexpr int MQ = 128;         // GEMM1 M = GEMM2 K: the points, padded
    static constexpr int KC = 64;          // GEMM2 K per chunk (two chunks through one G buffer)
    static constexpr int NT = 256;         // threads (eight warps, two per TMEM lane quarter)
    static constexpr int kTmemCols = 128;  // D1 at columns [0, 32), D2 at [64, 128)
    static constexpr int kD2 = 64;
    // shared memory (bytes from a 1024-aligned base).  The operator twice, as
    // K-major 128-byte swizzled operands (TF32 MN-major operands would need the
    // 32-byte-granule swizzle instead, so GEMM2 gets its own copy, B^T):
    //   Bop [128 q][64 b] (GEMM1's A), Bt [64 b][128 q] (GEMM2's B), hi and lo each
    static constexpr int kBopAtom = MQ * 128;           // 16384: a 32-wide k atom of Bop over 128 rows
    static constexpr int kBtAtom = NB * 128;            // 8192: a 32-wide k atom of Bt over 64 rows
    static constexpr int kBopHi = 0, kBopLo = 2 * kBopAtom;
    static constexpr int kBtHi = 4 * kBopAtom, kBtLo = kBtHi + 4 * kBtAtom;
    static constexpr int kOpBytes = 4 * kBopAtom + 8 * kBtAtom;  // 131072: one bulk copy
    static constexpr int kUopAtom = N1 * 128;           // 4096
    static constexpr int kUopHi = kOpBytes, kUopLo = kUopHi + 2 * kUopAtom;  // [32 c][64 b] each
    // G: [128 rows][KC points] per chunk; rows 96..127 are never written (their
    // outputs are ignored), so the k atoms are packed at 12 row groups (12288
    // bytes) and those rows read into the next atom (past the last one, into Fh)
    static constexpr int kGAtom = 12 * 1024;
    static constexpr int kGHi = kUopLo + 2 * kUopAtom, kGLo = kGHi + 2 * kGAtom;
    static constexpr int kFh = kGLo + 2 * kGAtom;       // face fluxes [E][6][5][FS] FP32
    static constexpr int kFhBytes = ((E * 30 * FS * 4 + 15) / 16) * 16;
    static constexpr int kRec = kFh + kFhBytes;         // face records [E][6]
    static constexpr int kMeta = kRec + E * 6 * 48;     // per element: JD[9], eref, hr, pref (FP32) [E][12]
    static constexpr int kCls = kMeta + E * 12 * 4;     // geometry class [E]
    static constexpr int kBar = ((kCls + E * 4 + 7) / 8) * 8;  // mbarriers: operator, GEMM1, GEMM2
    static constexpr int kSlot = kBar + 3 * 8;          // TMEM base address
    static constexpr int kBytes = kSlot + 16;
    static constexpr size_t kSmem = kBytes + 1024;      // + alignment slack
    // epilogue buffers over regions that are free by then
    static constexpr int kPart = kGHi;                  // FP32 [3][C][PS] direction partials (G is dead)
    static constexpr int PS = NB + 1;
    static constexpr int kRes = kPart + ((3 * C * PS * 4 + 15) / 16) * 16;  // FP64 [C][PS] residual
    static constexpr int kLift = kUopHi;                // FP32 [E][6][5][N*N] face lifts (Uop is dead)
    static_assert(kRes + C * PS * 8 <= kFh, "epilogue buffers must fit in the G region");
    static_assert(kLift + E * 30 * N * N * 4 <= kGHi, "lift buffer must fit in the Uop region");
    static_assert(kGLo + kGAtom + 16 * 1024 <= kBytes, "the last G atom's unused rows must stay inside shared memory");
    static_assert(kSmem <= 227 * 1024, "tensor-core stage kernel exceeds 227 KB of shared memory");
};

// host: TF32 rounding of cvt.rna.tf32.f32 (to nearest, ties away from zero)
inline float tf32_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u = (u + 0x1000u) & ~0x1FFFu;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// host: the operator B[q][b] of order P -- q over the (p+2)^3 volume points
// (q = qx + M qy + M^2 qz, zero rows past them), b over the (p+1)^3 basis
// functions (b = bx + N by + N^2 bz), B = B1[qx][bx] B1[qy][by] B1[qz][bz] --
// as TF32 hi and lo, in the swizzled layouts of TcCfg: Bop [q][b] then
// Bt [b][q] (kOpBytes, one bulk copy).  B1[q * N + b] is the 1D basis at the
// GL points.
template <int P>
void tc_operator_table(const double* B1, float* out)
{
    using K = TcCfg<P>;
    constexpr int N = K::N, M = K::M;
    for (int i = 0; i < K::kOpBytes / 4; ++i) out[i] = 0.f;
    for (int q = 0; q < K::NQ; ++q)
        for (int b = 0; b < K::NB; ++b) {
            const double v = B1[(q % M) * N + b % N] * B1[((q / M) % M) * N + (b / N) % N] * B1[(q / (M * M)) * N + b / (N * N)];
            const float hi = tf32_host(static_cast<float>(v));
            const float lo = tf32_host(static_cast<float>(v - static_cast<double>(hi)));
            const uint32_t o1 = tc::sw128(q, b, K::kBopAtom), o2 = tc::sw128(b, q, K::kBtAtom);
            out[(K::kBopHi + o1) / 4] = hi;
            out[(K::kBopLo + o1) / 4] = lo;
            out[(K::kBtHi + o2) / 4] = hi;
            out[(K::kBtLo + o2) / 4] = lo;
        }
}

// the kernel
template <int P>
__global__ void __launch_bounds__(TcCfg<P>::NT, 1) tc_stage_kernel(StageArgs a)
{
    using K = TcCfg<P>;
    constexpr int N = K::N, M = K::M, NB = K::NB, NQ = K::NQ, NF = K::NF, FS = K::FS, E = K::E, C = K::C;
    constexpr int N2 = N * N, PS = K::PS;
    constexpr long long kWait = 2000000000ll;  // ~1 s at 2 GHz
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = tc::smem_u32(smem_raw);
    const uint32_t sbase = (raw + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
    unsigned char* sm = smem_raw + (sbase - raw);
    float* Fh = reinterpret_cast<float*>(sm + K::kFh);
    FaceRec* sRec = reinterpret_cast<FaceRec*>(sm + K::kRec);
    float* sMeta = reinterpret_cast<float*>(sm + K::kMeta);
    int* sCls = reinterpret_cast<int*>(sm + K::kCls);
    float* Part = reinterpret_cast<float*>(sm + K::kPart);
    double* Res = reinterpret_cast<double*>(sm + K::kRes);
    float* Lift = reinterpret_cast<float*>(sm + K::kLift);
    const uint32_t barOp = sbase + K::kBar, bar1 = barOp + 8, bar2 = barOp + 16;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + K::kSlot);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float* __restrict__ Bt = a.tab.Bf;
    const float* __restrict__ Wt = a.tab.Wf;
    const float* __restrict__ Dn = a.tab.Dn;
    const double* __restrict__ Mi = a.tab.Minv;
    const float gamma = float(a.gamma);
    const int ntiles = (a.ne - a.e_begin + E - 1) / E;
    const bool need_acc = a.mode == kModeRK2 || a.mode == kModeRK3 || a.mode == kModeRK4;
    const bool need_u0 = a.mode >= kModeRK1;
    unsigned status = 0;

    if (warp == 0) {
        tc::tmem_alloc(sbase + K::kSlot, K::kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(barOp, 1);
        tc::mbar_init(bar1, 1);
        tc::mbar_init(bar2, 1);
        tc::mbar_fence_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *slot;
    const uint32_t d1 = tmem, d2 = tmem + K::kD2;
    if (tid == 0 && (int)blockIdx.x < ntiles) {
        tc::mbar_expect_tx(barOp, K::kOpBytes);
        tc::bulk_g2s(sbase, a.tcop, K::kOpBytes, barOp);
    }
    // the state (and the RK operands) of tile t into L2 ahead of their plain loads
    auto prefetch_tile = [&](int t) {
        if (t >= ntiles) return;
        const int e0 = a.e_begin + t * E, nel = min(E, a.ne - e0);
        const int lines = nel * 5 * NB * 8 / 128;  // 20 per element
        const size_t off = (size_t)e0 * 5 * NB;
        for (int i = tid; i < 3 * lines; i += K::NT) {
            const int k = i / lines, l = i - k * lines;
            const double* src = k == 0 ? a.Us : (k == 1 ? (need_u0 ? a.U0 : nullptr) : (need_acc ? a.acc : nullptr));
            if (src) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(src + off + l * 16));
        }
    };
    prefetch_tile(blockIdx.x);
    bool alive = __syncthreads_and(tc::mbar_wait(barOp, 0, kWait));
    if (!alive) status |= kStatusTimeout;
    uint32_t ph1 = 0, ph2 = 0;
    for (int t = blockIdx.x; t < ntiles && alive; t += gridDim.x) {
        const int e0 = a.e_begin + t * E, nel = min(E, a.ne - e0);
        prefetch_tile(t + gridDim.x);
        // ---- face records and geometry of the tile ----
        for (int i = tid; i < E * 6 * 3; i += K::NT) {  // 16-byte pieces of the records
            const int e = i / 18;
            const int ge = min(e0 + e, a.ne - 1);
            reinterpret_cast<int4*>(sRec)[i] = reinterpret_cast<const int4*>(a.frec + (size_t)ge * 6)[i - e * 18];
        }
        if (tid < E) {
            const int ge = min(e0 + tid, a.ne - 1);
            const int cls = a.geo_class[ge];
            const GeoDev& g = a.geo[cls];
            sCls[tid] = cls;
            float* mt = sMeta + tid * 12;
#pragma unroll
            for (int k = 0; k < 9; ++k) mt[k] = float(g.JD[k]);
            mt[9] = float(g.eref);
            mt[10] = float(a.gamma * g.eref);
            mt[11] = float((a.gamma - 1.0) * g.eref);
        }
        __syncthreads();
        // ---- the state as GEMM1's B operand (rows c = 5 e + v, K = b), hi / lo ----
        for (int i = tid; i < K::N1 * NB; i += K::NT) {
            const int c = i / NB, b = i - c * NB, e = c / 5, v = c - 5 * e;
            float hi = 0.f, lo = 0.f;
            if (c < C && e < nel) {
                const double x = a.Us[(size_t)e0 * 5 * NB + i] - (v == 4 ? a.geo[sCls[e]].eref : 0.0);
                hi = tc::tf32(float(x));
                lo = tc::tf32(float(x - double(hi)));
            }
            const uint32_t off = tc::sw128(c, b, K::kUopAtom);
            *reinterpret_cast<float*>(sm + K::kUopHi + off) = hi;
            *reinterpret_cast<float*>(sm + K::kUopLo + off) = lo;
        }
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            // GEMM1: D1[q][c] = sum_b B[q][b] U[c][b]; lo*hi, hi*lo, hi*hi
            constexpr uint32_t id1 = tc::idesc_tf32(128, K::N1, 0);
#pragma unroll
            for (int s = 0; s < 3; ++s) {
                const uint32_t ab = sbase + (s == 0 ? K::kBopLo : K::kBopHi);
                const uint32_t bb = sbase + (s == 1 ? K::kUopLo : K::kUopHi);
#pragma unroll
                for (int kk = 0; kk < NB / 8; ++kk) {
                    const uint64_t ad = tc::sdesc(ab + (kk >> 2) * K::kBopAtom + (kk & 3) * 32, 16, 1024);
                    const uint64_t bd = tc::sdesc(bb + (kk >> 2) * K::kUopAtom + (kk & 3) * 32, 16, 1024);
                    tc::mma_tf32(d1, ad, bd, id1, (s > 0 || kk > 0) ? 1u : 0u);
                }
            }
            tc::mma_commit(bar1);
        }
        // the six faces' fluxes of the face kernel (the listed side reads its own
        // point order, the other side through the face-point permutation)
        {
            const float* gF = reinterpret_cast<const float*>(a.fflux);
            for (int i = tid; i < E * 6 * NF; i += K::NT) {
                const int c = i % NF, f = (i / NF) % 6, e = i / (6 * NF);
                if (e >= nel) continue;
                const FaceRec& rec = sRec[e * 6 + f];
                const int pc = ((rec.pad >> 30) & 1) ? c : a.cmap[(rec.info >> 4) * NF + c];
                const float* src = gF + (size_t)(rec.pad & 0x3fffffff) * 5 * NF + pc;
                float* dst = Fh + (e * 6 + f) * 5 * FS + c;
#pragma unroll
                for (int v = 0; v < 5; ++v) cp_async4(dst + v * FS, src + v * NF);
            }
            cp_async_commit();
        }
        // ---- the flux at every point: D1 -> G (GEMM2's A operand) ----
        if (!__syncthreads_and(tc::mbar_wait(bar1, ph1, kWait))) {
            status |= kStatusTimeout;
            alive = false;
            break;
        }
        ph1 ^= 1;
        tc::tc_fence_after();
        const int qt = warp & 3, fhalf = warp >> 2;
        const int q = qt * 32 + lane;
        const int chunk = qt >> 1;        // this warp's points fall in GEMM2's K chunk 0 (q < 64) or 1
        const int ql = q - chunk * K::KC;  // point within the chunk
        float G[3][15];                    // this thread's fluxes: 3 elements x (d, v)
        {
            float u[32];  // all 32 columns (aligned loads); this half's elements start at column 15 fhalf
            const uint32_t lrow = d1 + (static_cast<uint32_t>(qt * 32) << 16);
            tc::tmem_ld16(lrow, u);
            tc::tmem_ld16(lrow + 16, u + 16);
            tc::tmem_wait_ld();
            const int qx = q % M, qy = (q / M) % M, qz = q / (M * M);
            const float wq = q < NQ ? Wt[qx] * Wt[qy] * Wt[qz] : 0.f;
#pragma unroll
            for (int ee = 0; ee < 3; ++ee) {
                const int e = fhalf * 3 + ee;
                if (q < NQ && e < nel) {
                    const float* mt = sMeta + e * 12;
                    float U[5], F[15];
#pragma unroll
                    for (int v = 0; v < 5; ++v) U[v] = fhalf ? u[15 + ee * 5 + v] : u[ee * 5 + v];
                    const float p = dgp::interior_flux_r1<float, true>(gamma, U, F, mt[10]);
                    if (!(U[0] > 0.f)) status |= kStatusRho;
                    if (!(p + mt[11] > 0.f)) status |= kStatusPressure;
                    if (U[0] != U[0] || p != p) status |= kStatusNaN;
#pragma unroll
                    for (int v = 0; v < 5; ++v)
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            G[ee][d * 5 + v] = (F[v] * mt[d * 3 + 0] + F[5 + v] * mt[d * 3 + 1] + F[10 + v] * mt[d * 3 + 2]) * wq;
                } else {
#pragma unroll
                    for (int k = 0; k < 15; ++k) G[ee][k] = 0.f;
                }
            }
        }
        // G of one chunk into the buffer: rows 32 d + 5 e + v, K = the point within the chunk
        auto store_G = [&]() {
#pragma unroll
            for (int ee = 0; ee < 3; ++ee) {
                const int e = fhalf * 3 + ee;
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int v = 0; v < 5; ++v) {
                        const float g = G[ee][d * 5 + v];
                        const float hi = tc::tf32(g), lo = tc::tf32(g - hi);
                        const uint32_t off = tc::sw128(32 * d + 5 * e + v, ql, K::kGAtom);
                        *reinterpret_cast<float*>(sm + K::kGHi + off) = hi;
                        *reinterpret_cast<float*>(sm + K::kGLo + off) = lo;
                    }
            }
        };
        // GEMM2 over chunk ch: H[r][b] += sum_{q in chunk} G[r][q] Bt[b][q]
        auto issue_gemm2 = [&](int ch) {
            constexpr uint32_t id2 = tc::idesc_tf32(128, NB, 0);
#pragma unroll
            for (int s = 0; s < 3; ++s) {
                const uint32_t ab = sbase + (s == 0 ? K::kGLo : K::kGHi);
                const uint32_t bb = sbase + (s == 1 ? K::kBtLo : K::kBtHi);
#pragma unroll
                for (int kl = 0; kl < K::KC / 8; ++kl) {
                    const int kk = ch * (K::KC / 8) + kl;
                    const uint64_t ad = tc::sdesc(ab + (kl >> 2) * K::kGAtom + (kl & 3) * 32, 16, 1024);
                    const uint64_t bd = tc::sdesc(bb + (kk >> 2) * K::kBtAtom + (kk & 3) * 32, 16, 1024);
                    tc::mma_tf32(d2, ad, bd, id2, (ch > 0 || s > 0 || kl > 0) ? 1u : 0u);
                }
            }
            tc::mma_commit(bar2);
        };
        if (chunk == 0) store_G();
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            issue_gemm2(0);
        }
        // the first chunk must be consumed before the second overwrites the buffer
        if (!__syncthreads_and(tc::mbar_wait(bar2, ph2, kWait))) {
            status |= kStatusTimeout;
            alive = false;
            break;
        }
        ph2 ^= 1;
        tc::tc_fence_after();
        if (chunk == 1) store_G();
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            issue_gemm2(1);
        }
        // ---- face lifts (FP32) while GEMM2 runs, into the Uop region ----
        cp_async_wait_all();
        __syncthreads();
        for (int t2 = tid; t2 < E * 30; t2 += K::NT) {
            const int v = t2 % 5, f = (t2 / 5) % 6, e = t2 / 30;
            if (e >= nel) continue;
            const float* Fq = Fh + ((e * 6 + f) * 5 + v) * FS;
            const float sgn = ((sRec[e * 6 + f].info >> 3) & 1) ? -1.f : 1.f;
            float tmp[M][N];
#pragma unroll
            for (int t1 = 0; t1 < M; ++t1)
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) {
                    float s = 0.f;
#pragma unroll
                    for (int t0 = 0; t0 < M; ++t0) s += Bt[t0 * N + b0] * Fq[t1 * M + t0];
                    tmp[t1][b0] = s;
                }
            float* Lf = Lift + ((e * 6 + f) * 5 + v) * N2;
#pragma unroll
            for (int b1 = 0; b1 < N; ++b1)
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) {
                    float s = 0.f;
#pragma unroll
                    for (int t1 = 0; t1 < M; ++t1) s += Bt[t1 * N + b1] * tmp[t1][b0];
                    Lf[b1 * N + b0] = sgn * s;
                }
        }
        // ---- Delta_d^T along each axis (FP32), one warp per direction and half ----
        if (!__syncthreads_and(tc::mbar_wait(bar2, ph2, kWait))) {
            status |= kStatusTimeout;
            alive = false;
            break;
        }
        ph2 ^= 1;
        tc::tc_fence_after();
        {
            const int d = warp & 3, half = warp >> 2;
            if (d < 3) {
                const uint32_t row = d2 + (static_cast<uint32_t>(d * 32) << 16);
                float h[32];
                if (d < 2) {
                    tc::tmem_ld16(row + half * 32, h);
                    tc::tmem_ld16(row + half * 32 + 16, h + 16);
                } else {
#pragma unroll
                    for (int bz = 0; bz < 4; ++bz) {
                        float r8[8];
                        tc::tmem_ld8(row + bz * 16 + half * 8, r8);
#pragma unroll
                        for (int k = 0; k < 8; ++k) h[bz * 8 + k] = r8[k];
                    }
                }
                tc::tmem_wait_ld();
                const int c = lane;
                if (c < C && c / 5 < nel) {
                    float* out = Part + (d * C + c) * PS;
                    if (d == 0) {
                        // h[(bz - 2 half) * 16 + by * 4 + bx]
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
#pragma unroll
                            for (int bx = 0; bx < N; ++bx) {
                                float s = 0.f;
#pragma unroll
                                for (int i = 0; i < N; ++i) s += Dn[i * N + bx] * h[j * 4 + i];
                                out[half * 32 + j * 4 + bx] = s;
                            }
                        }
                    } else if (d == 1) {
#pragma unroll
                        for (int bzl = 0; bzl < 2; ++bzl)
#pragma unroll
                            for (int bx = 0; bx < N; ++bx)
#pragma unroll
                                for (int by = 0; by < N; ++by) {
                                    float s = 0.f;
#pragma unroll
                                    for (int i = 0; i < N; ++i) s += Dn[i * N + by] * h[bzl * 16 + i * 4 + bx];
                                    out[half * 32 + bzl * 16 + by * 4 + bx] = s;
                                }
                    } else {
                        // h[bz * 8 + byl * 4 + bx], by = 2 half + byl
#pragma unroll
                        for (int k = 0; k < 8; ++k)
#pragma unroll
                            for (int bz = 0; bz < N; ++bz) {
                                float s = 0.f;
#pragma unroll
                                for (int i = 0; i < N; ++i) s += Dn[i * N + bz] * h[i * 8 + k];
                                out[bz * 16 + half * 8 + k] = s;
                            }
                    }
                }
            }
        }
        tc::tc_fence_before();
        __syncthreads();
        // ---- residual (FP64): directions + face lifts ----
        for (int i = tid; i < C * NB; i += K::NT) {
            const int c = i / NB, b = i - c * NB, e = c / 5, v = c - 5 * e;
            if (e >= nel) continue;
            double s = double(Part[c * PS + b]) + double(Part[(C + c) * PS + b]) + double(Part[(2 * C + c) * PS + b]);
            const int bc[3] = {b % N, (b / N) % N, b / N2};
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                const int ax = face_axis(f), sidx = face_side(f) ? N - 1 : 0;
                if (bc[ax] == sidx) {
                    const int b0 = ax == 0 ? bc[1] : bc[0];
                    const int b1 = ax == 2 ? bc[1] : bc[2];
                    s += double(Lift[((e * 6 + f) * 5 + v) * N2 + b1 * N + b0]);
                }
            }
            Res[c * PS + b] = s;
        }
        __syncthreads();
        if (a.mode == kModeResidual) {
            for (int i = tid; i < nel * 5 * NB; i += K::NT) {
                const int c = i / NB, b = i - c * NB;
                a.out[(size_t)e0 * 5 * NB + i] = Res[c * PS + b];
            }
            __syncthreads();
            continue;
        }
        // ---- inverse mass (FP64): x and y passes in place, z pass with the update ----
        for (int i = tid; i < nel * 5 * N2; i += K::NT) {
            const int c = i / N2, r = i - c * N2;
            double* rr = Res + c * PS + r * N;  // pencil along x at (by, bz) = r
            double t4[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t4[k] = rr[k];
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t4[k];
                rr[j] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < nel * 5 * N2; i += K::NT) {
            const int c = i / N2, r = i - c * N2, bx = r % N, bz = r / N;
            double* rr = Res + c * PS + bz * N2 + bx;  // pencil along y
            double t4[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t4[k] = rr[k * N];
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t4[k];
                rr[j * N] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < nel * 5 * N2; i += K::NT) {
            const int c = i / N2, bxy = i - c * N2, e = c / 5;
            const GeoDev& gg = a.geo[sCls[e]];
            const double scale = a.dt * gg.dtf * gg.inv_djac;
            const double* rr = Res + c * PS + bxy;  // pencil along z
            double t4[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t4[k] = rr[k * N2];
            const size_t gbase = (size_t)e0 * 5 * NB + (size_t)c * NB + bxy;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[j * N + k] * t4[k];
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
    // a CTA that gave up waiting for the operator may still have its copy in
    // flight: wait for it (bounded) before the shared memory goes away
    if (!alive && tid == 0) (void)tc::mbar_wait(barOp, 0, kWait);
    cp_async_wait_all();
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, K::kTmemCols);
    }
    if (status) atomicOr(a.status, status);
}

template <int P>
cudaError_t launch_tc_stage(const StageArgs& a, int grid, cudaStream_t s)
{
    tc_stage_kernel<P><<<grid, TcCfg<P>::NT, TcCfg<P>::kSmem, s>>>(a);
    return cudaGetLastError();
}

// the tensor-core kernel as a launch variant of order P (FP32 residual, with
// the face kernel before it; the option bits besides TC describe what it
// shares with the unfused single-buffer face-flux variants)
template <int P>
StageVariant make_tc_variant()
{
    using K = TcCfg<P>;
    StageVariant v{K::E, K::NT, 1, 1, kUF | kSB | kFX | kTC, K::kSmem, (const void*)tc_stage_kernel<P>,
                   launch_tc_stage<P>, (const void*)face_flux_kernel<P, float, false>, face_smem_bytes<P, float>(),
                   kFaceThreads, launch_face_kernel<P, float, false>, face_batch<P, float>()};
    return v;
}

}  // namespace dgk
