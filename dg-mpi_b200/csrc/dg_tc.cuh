// dg_tc.cuh -- the tensor-core stage kernel (sm_100a, tcgen05): the volume
// integral of the FP32 residual as split-BF16 products on the 5th-generation
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
// Per tile of E elements (grid-stride over tiles):
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
//          stored once, serves both GEMMs: K-major as GEMM1's A, MN-major as
//          GEMM2's B;
//   then, on the CUDA cores, Delta_d^T along each axis (FP32), the face lift of
//   the face kernel's fluxes (FP32), the sum into the FP64 residual, the
//   Kronecker inverse mass and the RK stage update in FP64.
// Split products (BF16x6): every operand x (FP32) is stored as three BF16
// parts x = x0 + x1 + x2 (8 significant bits each: exact for an FP32 value)
// and each GEMM accumulates the six products xi * yj with i + j <= 2, the
// small ones first; what is left out (i + j >= 3) is below 2^-23 of the
// product, so the GEMMs keep FP32's accuracy.  BF16 MMAs run at twice the
// TF32 rate: six of them cost what the three products of TF32x3 cost, and
// TF32x3 (22-bit operands) measured 4-5x less accurate than FP32 here.
// The state enters as U - E_ref in its energy (the FP32 residual's energy
// reference, see dgp::interior_flux_r1).
//
// Two CTAs per SM (about 100 KB of shared memory and at most 128 registers
// per thread each) hide each other's waits: the operator (48 KB), the
// state's three parts, and GEMM2's A operand in two chunks of 64 points (the
// points of lane quarters 0-1, then 2-3: the second chunk is written once the
// first has been multiplied, the face lifts run in between).  The next
// tile's face records are bulk-copied into shared memory ahead of use; its
// state, RK operands and face fluxes are prefetched into L2.  Every wait on
// an mbarrier is bounded (clock64); a wait that gives up sets
// kStatusTimeout, the CTA stops, waits (bounded) for its copies in flight,
// releases its TMEM and returns.  No multicast, no peer memory: every
// operand is in this CTA's own shared memory.
//
// Shared-memory operands use the 128-byte swizzled canonical layout of the
// UMMA descriptors: atoms of 8 rows x 128 bytes (64 BF16 elements along the
// atom's row), 1024-byte aligned, with the 16-byte chunk index of a row XORed
// with the row's index within the atom.
#pragma once
#include <cuda_bf16.h>

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
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint32_t bar) { asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory"); }
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
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }

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

// D (TMEM, FP32) (+)= A (smem) * B (smem), kind::f16 with BF16 operands, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
// arrives on the mbarrier once every MMA issued so far by this thread is complete
__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

// TMEM -> registers: this warp's 32 lanes (lane quarter warp % 4), consecutive columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* r)
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

// x = x0 + x1 + x2 exactly, each part a BF16 (round to nearest even)
__device__ __forceinline__ void split3(float x, uint16_t (&p)[3])
{
    const __nv_bfloat16 b0 = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(b0);
    const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(b1);
    const __nv_bfloat16 b2 = __float2bfloat16_rn(r2);
    p[0] = __bfloat16_as_ushort(b0);
    p[1] = __bfloat16_as_ushort(b1);
    p[2] = __bfloat16_as_ushort(b2);
}

// ---- descriptors ----
// shared-memory matrix descriptor, 128-byte swizzle (layout type 2), version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}
// instruction descriptor of kind::f16 with BF16 A and B and FP32 accumulation:
// M rows, N columns, A K-major, B K-major (b_mn = 0) or MN-major (b_mn = 1)
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(b_mn) << 16) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// byte offset of element (row, k) of a two-byte operand in 128-byte swizzled
// atoms: 8-row groups at 1024 bytes, 64-element atoms along k at `katom` bytes
__host__ __device__ constexpr uint32_t sw128h(int row, int k, int katom)
{
    return static_cast<uint32_t>((k >> 6) * katom + (row >> 3) * 1024 + (row & 7) * 128 +
                                 ((((k & 63) >> 3) ^ (row & 7)) << 4) + (k & 7) * 2);
}

// the six products x_i * y_j (i + j <= 2), small ones first
__host__ __device__ constexpr int prod_a(int s) { return s == 0 ? 0 : s == 1 ? 1 : s == 2 ? 2 : s == 3 ? 0 : s == 4 ? 1 : 0; }
__host__ __device__ constexpr int prod_b(int s) { return s == 0 ? 2 : s == 1 ? 1 : s == 2 ? 0 : s == 3 ? 1 : s == 4 ? 0 : 0; }

}  // namespace tc

// ---- the kernel's configuration per order (p = 3: nb = 64, 125 volume points) ----
template <int P>
struct TcCfg;
template <>
struct TcCfg<3> {
    static constexpr int N = 4, M = 5, NB = 64, NQ = 125, NF = 25;
    static constexpr int E = 6;            // elements per tile
    static constexpr int C = 5 * E;        // (element, variable) columns of a tile (30)
    static constexpr int N1 = 32;          // GEMM1 N: the columns, padded to 32
    static constexpr int MQ = 128;         // GEMM1 M = GEMM2 K: the points, padded
    static constexpr int KC = 64;          // GEMM2 K per chunk: the points of two TMEM lane quarters
    static constexpr int NT = 256;         // threads (eight warps, two per TMEM lane quarter)
    static constexpr int MINB = 2;         // CTAs per SM (registers <= 128 per thread)
    static constexpr int FSTR = 128;       // FP32 elements per face in the face kernel's output (5 x 25, padded)
    // TMEM: each GEMM accumulates its hi * hi products and its five small
    // products (x_i y_j, 0 < i + j <= 2) in separate accumulators, added at
    // the read-out, so FP32 rounding of the large sum does not swallow the
    // small terms: D1 big / small at columns [0, 32) / [32, 64), D2 big /
    // small at [64, 128) / [128, 192)
    static constexpr int kTmemCols = 256;
    static constexpr int kD1s = 32, kD2 = 64, kD2s = 128;
    // shared memory (bytes from a 1024-aligned base)
    static constexpr int kOpPart = MQ * 128;             // [128 q][64 b] BF16, one 64-wide k atom: 16384
    static constexpr int kOp = 0, kOpBytes = 3 * kOpPart;
    static constexpr int kUopPart = N1 * 128;            // [32 c][64 b] BF16: 4096
    static constexpr int kUop = kOpBytes;
    // G: [128 rows][KC points] BF16 per part, one 64-wide k atom; rows 96..127
    // are never written (their outputs are ignored), so the parts are packed at
    // 12 row groups (12288 bytes) and those rows read into the next part (past
    // the last one, into the records after it)
    static constexpr int kGPart = 12 * 1024;
    static constexpr int kG = kUop + 3 * kUopPart;
    static constexpr int kRec = kG + 3 * kGPart;         // face records [2][E][6]
    static constexpr int kRecBytes = E * 6 * 48;
    static constexpr int kMeta = kRec + 2 * kRecBytes;   // per element: JD[9], eref, hr, pref (FP32) [2][E][12]
    static constexpr int kCls = kMeta + 2 * E * 12 * 4;  // geometry class [2][E]
    static constexpr int kBar = ((kCls + 2 * E * 4 + 7) / 8) * 8;  // mbarriers
    static constexpr int kNumBar = 5;  // operator, frec slot 0 / 1, GEMM1, GEMM2
    static constexpr int kSlot = kBar + kNumBar * 8;    // TMEM base address
    static constexpr int kBytes = ((kSlot + 16 + 15) / 16) * 16;
    static constexpr size_t kSmem = kBytes + 1024;      // + alignment slack
    // epilogue buffers over regions that are free by then
    static constexpr int PS = NB + 1;
    static constexpr int kPart = kG;                     // FP32 [3][C][PS]; FP64 residual [C][PS] over it (GEMM2 done)
    static constexpr int kLift = kUop;                   // FP32 [E][6][5][N*N] face lifts (GEMM1 done)
    static_assert(C * PS * 8 <= 3 * C * PS * 4, "the FP64 residual must fit over the direction partials");
    static_assert(kPart + 3 * C * PS * 4 <= kRec, "direction partials must fit in the G region");
    static_assert(kLift + E * 30 * N * N * 4 <= kG, "face lifts must fit in the Uop region");
    static_assert(kG + 2 * kGPart + 16 * 1024 <= kBytes, "the last G part's unused rows must stay inside shared memory");
    static_assert(kRec % 16 == 0 && kRecBytes % 16 == 0, "bulk-copy targets");
    static_assert((FSTR * 4) % 16 == 0 && FSTR >= 5 * NF, "face block stride");
    static_assert(MINB * (kSmem + 1024) <= 228 * 1024, "two CTAs per SM");
};

// host: FP32 -> BF16 bits, round to nearest even (finite values)
inline uint16_t bf16_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(u >> 16);
}
inline float bf16_value(uint16_t h)
{
    const uint32_t u = static_cast<uint32_t>(h) << 16;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// host: the operator B[q][b] of order P -- q over the (p+2)^3 volume points
// (q = qx + M qy + M^2 qz, zero rows past them), b over the (p+1)^3 basis
// functions (b = bx + N by + N^2 bz), B = B1[qx][bx] B1[qy][by] B1[qz][bz] --
// as three BF16 parts (B = B0 + B1 + B2 to 24 bits) in the swizzled layout of
// TcCfg (kOpBytes, one bulk copy).  B1[q * N + b] is the 1D basis at the GL
// points.
template <int P>
void tc_operator_table(const double* B1, uint16_t* out)
{
    using K = TcCfg<P>;
    constexpr int N = K::N, M = K::M;
    for (int i = 0; i < K::kOpBytes / 2; ++i) out[i] = 0;
    for (int q = 0; q < K::NQ; ++q)
        for (int b = 0; b < K::NB; ++b) {
            const double v = B1[(q % M) * N + b % N] * B1[((q / M) % M) * N + (b / N) % N] * B1[(q / (M * M)) * N + b / (N * N)];
            const float vf = static_cast<float>(v);
            const uint16_t h0 = bf16_host(vf);
            const float r1 = vf - bf16_value(h0);
            const uint16_t h1 = bf16_host(r1);
            const uint16_t h2 = bf16_host(r1 - bf16_value(h1));
            const uint32_t o = tc::sw128h(q, b, K::kOpPart) / 2;
            out[o] = h0;
            out[K::kOpPart / 2 + o] = h1;
            out[K::kOpPart + o] = h2;
        }
}

// the flux at point q for the three elements of half FH of a tile, written
// as GEMM2's A operand: rows 32 d + 5 e + v, column ql (the point within the
// chunk), three BF16 parts.  u: D1 row of this lane (all 32 columns).
template <int P, int FH>
__device__ __forceinline__ void tc_flux_half(const float (&u)[32], int q, int ql, int nel, const float* __restrict__ mtab,
                                             float gamma, float wq, unsigned char* gbase, unsigned& status)
{
    using K = TcCfg<P>;
    const uint32_t kc = static_cast<uint32_t>((ql >> 3) & 7), kb = static_cast<uint32_t>((ql & 7) * 2);
#pragma unroll
    for (int ee = 0; ee < 3; ++ee) {
        const int e = FH * 3 + ee;
        float G[15];
        if (q < K::NQ && e < nel) {
            const float* mt = mtab + e * 12;
            float U[5], F[15];
#pragma unroll
            for (int v = 0; v < 5; ++v) U[v] = u[FH * 15 + ee * 5 + v];
            const float p = dgp::interior_flux_r1<float, true>(gamma, U, F, mt[10]);
            if (!(U[0] > 0.f)) status |= kStatusRho;
            if (!(p + mt[11] > 0.f)) status |= kStatusPressure;
            if (U[0] != U[0] || p != p) status |= kStatusNaN;
#pragma unroll
            for (int v = 0; v < 5; ++v)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    G[d * 5 + v] = (F[v] * mt[d * 3 + 0] + F[5 + v] * mt[d * 3 + 1] + F[10 + v] * mt[d * 3 + 2]) * wq;
        } else {
#pragma unroll
            for (int k = 0; k < 15; ++k) G[k] = 0.f;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const int row = 32 * d + 5 * (FH * 3 + ee) + v;  // compile time
                uint16_t parts[3];
                tc::split3(G[d * 5 + v], parts);
                unsigned char* p0 = gbase + (row >> 3) * 1024 + (row & 7) * 128 + ((kc ^ (row & 7)) << 4) + kb;
#pragma unroll
                for (int k = 0; k < 3; ++k) *reinterpret_cast<uint16_t*>(p0 + k * K::kGPart) = parts[k];
            }
    }
}

// the kernel
template <int P>
__global__ void __launch_bounds__(TcCfg<P>::NT, TcCfg<P>::MINB) tc_stage_kernel(StageArgs a)
{
    using K = TcCfg<P>;
    constexpr int N = K::N, M = K::M, NB = K::NB, NQ = K::NQ, NF = K::NF, E = K::E, C = K::C;
    constexpr int N2 = N * N, PS = K::PS, FSTR = K::FSTR;
    constexpr long long kWait = 2000000000ll;  // ~1 s at 2 GHz
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = tc::smem_u32(smem_raw);
    const uint32_t sbase = (raw + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
    unsigned char* sm = smem_raw + (sbase - raw);
    float* Part = reinterpret_cast<float*>(sm + K::kPart);
    double* Res = reinterpret_cast<double*>(sm + K::kPart);  // over Part, after the sum
    float* Lift = reinterpret_cast<float*>(sm + K::kLift);
    const uint32_t barOp = sbase + K::kBar, barR0 = barOp + 8, bar1 = barOp + 24, bar2 = barOp + 32;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + K::kSlot);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float* __restrict__ Bt = a.tab.Bf;
    const float* __restrict__ Wt = a.tab.Wf;
    const float* __restrict__ Dn = a.tab.Dn;
    const double* __restrict__ Mi = a.tab.Minv;
    const float* __restrict__ gF = reinterpret_cast<const float*>(a.fflux);
    const float gamma = float(a.gamma);
    const int ntiles = (a.ne - a.e_begin + E - 1) / E;
    const int nt = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;  // this CTA's tiles
    const bool need_acc = a.mode == kModeRK2 || a.mode == kModeRK3 || a.mode == kModeRK4;
    const bool need_u0 = a.mode >= kModeRK1;
    unsigned status = 0;

    auto tile_e0 = [&](int j) { return a.e_begin + ((int)blockIdx.x + j * (int)gridDim.x) * E; };
    auto tile_nel = [&](int j) { return min(E, a.ne - tile_e0(j)); };
    auto recs = [&](int j) { return reinterpret_cast<const FaceRec*>(sm + K::kRec + (j & 1) * K::kRecBytes); };
    auto meta = [&](int j) { return reinterpret_cast<float*>(sm + K::kMeta + (j & 1) * E * 12 * 4); };
    auto cls = [&](int j) { return reinterpret_cast<int*>(sm + K::kCls + (j & 1) * E * 4); };

    if (warp == 0) {
        tc::tmem_alloc(sbase + K::kSlot, K::kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < K::kNumBar; ++i) tc::mbar_init(barOp + 8 * i, 1);
        tc::mbar_fence_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *slot;
    const uint32_t d1 = tmem, d1s = tmem + K::kD1s, d2 = tmem + K::kD2, d2s = tmem + K::kD2s;

    // face records of tile j into slot j & 1 (thread 0)
    bool pend[2] = {false, false};
    uint32_t pph[2] = {0, 0};
    auto load_recs = [&](int j) {
        const uint32_t bytes = tile_nel(j) * 6 * 48;
        const uint32_t bar = barR0 + 8 * (j & 1);
        tc::mbar_expect_tx(bar, bytes);
        tc::bulk_g2s(sbase + K::kRec + (j & 1) * K::kRecBytes, a.frec + (size_t)tile_e0(j) * 6, bytes, bar);
        pend[j & 1] = true;
        pph[j & 1] = (j >> 1) & 1;
    };
    // waits for phase `parity` of `bar` on every thread; false (uniformly) if it gave up
    auto wait_all = [&](uint32_t bar, uint32_t parity) {
        const bool ok = __syncthreads_and(tc::mbar_wait(bar, parity, kWait));
        if (!ok) status |= kStatusTimeout;
        return ok;
    };
    // the state of tile j and its RK operands into L2 ahead of their plain loads
    auto prefetch_state = [&](int j) {
        const int lines = tile_nel(j) * 5 * NB * 8 / 128;
        const size_t off = (size_t)tile_e0(j) * 5 * NB;
        for (int i = tid; i < 3 * lines; i += K::NT) {
            const int k = i / lines;
            const double* src = k == 0 ? a.Us : (k == 1 ? (need_u0 ? a.U0 : nullptr) : (need_acc ? a.acc : nullptr));
            if (src) tc::prefetch_l2(src + off + (i - k * lines) * 16);
        }
    };
    // the face fluxes of tile j (its records have landed) into L2
    auto prefetch_faces = [&](int j) {
        const FaceRec* r = recs(j);
        const int nel = tile_nel(j);
        for (int i = tid; i < nel * 6 * 4; i += K::NT)
            tc::prefetch_l2(gF + (size_t)(r[i >> 2].pad & 0x3fffffff) * FSTR + (i & 3) * 32);
    };

    bool alive = nt > 0;
    uint32_t ph1 = 0, ph2 = 0;
    if (alive) {
        if (tid == 0) {
            tc::mbar_expect_tx(barOp, K::kOpBytes);
            tc::bulk_g2s(sbase + K::kOp, a.tcop, K::kOpBytes, barOp);
            load_recs(0);
        }
        prefetch_state(0);
        alive = wait_all(barOp, 0);
    }
    for (int j = 0; j < nt && alive; ++j) {
        const int nel = tile_nel(j), e0 = tile_e0(j);
        // ---- this tile's records, the next tile's in flight ----
        if (!(alive = wait_all(barR0 + 8 * (j & 1), (j >> 1) & 1))) break;
        if (tid == 0) {
            pend[j & 1] = false;
            if (j + 1 < nt) load_recs(j + 1);
        }
        const FaceRec* r = recs(j);
        prefetch_faces(j);
        if (j + 1 < nt) prefetch_state(j + 1);
        if (tid < E) {
            const int c0 = r[min(tid, nel - 1) * 6].cls;
            const GeoDev& g = a.geo[c0];
            cls(j)[tid] = c0;
            float* mt = meta(j) + tid * 12;
#pragma unroll
            for (int k = 0; k < 9; ++k) mt[k] = float(g.JD[k]);
            mt[9] = float(g.eref);
            mt[10] = float(a.gamma * g.eref);
            mt[11] = float((a.gamma - 1.0) * g.eref);
        }
        __syncthreads();
        // ---- the state as GEMM1's B operand (rows c = 5 e + v, K = b), three parts ----
        {
            for (int i = tid; i < K::N1 * NB; i += K::NT) {
                const int c = i / NB, b = i - c * NB, e = c / 5, v = c - 5 * e;
                uint16_t parts[3] = {0, 0, 0};
                if (c < C && e < nel) {
                    const double x = a.Us[(size_t)e0 * 5 * NB + i] - (v == 4 ? a.geo[cls(j)[e]].eref : 0.0);
                    tc::split3(float(x), parts);
                }
                unsigned char* p0 = sm + K::kUop + tc::sw128h(c, b, K::kUopPart);
#pragma unroll
                for (int k = 0; k < 3; ++k) *reinterpret_cast<uint16_t*>(p0 + k * K::kUopPart) = parts[k];
            }
        }
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            constexpr uint32_t id1 = tc::idesc_bf16(128, K::N1, 0);
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const uint32_t ab = sbase + K::kOp + tc::prod_a(s) * K::kOpPart;
                const uint32_t bb = sbase + K::kUop + tc::prod_b(s) * K::kUopPart;
                const bool big = s == 5;
#pragma unroll
                for (int kk = 0; kk < NB / 16; ++kk)
                    tc::mma_bf16(big ? d1 : d1s, tc::sdesc(ab + kk * 32, 16, 1024), tc::sdesc(bb + kk * 32, 16, 1024),
                                 id1, ((big ? 0 : s) > 0 || kk > 0) ? 1u : 0u);
            }
            tc::mma_commit(bar1);
        }
        if (!(alive = wait_all(bar1, ph1))) break;
        ph1 ^= 1;
        tc::tc_fence_after();
        // ---- fluxes: D1 -> G in two chunks of points (lane quarters 0-1, then 2-3) ----
        const int qt = warp & 3, fhalf = warp >> 2;
        const int q = qt * 32 + lane, ql = q & (K::KC - 1);
        float u[32];
        {
            const uint32_t lrow = static_cast<uint32_t>(qt * 32) << 16;
            float us[32];
            tc::tmem_ld16(d1 + lrow, u);
            tc::tmem_ld16(d1 + lrow + 16, u + 16);
            tc::tmem_ld16(d1s + lrow, us);
            tc::tmem_ld16(d1s + lrow + 16, us + 16);
            tc::tmem_wait_ld();
#pragma unroll
            for (int k = 0; k < 32; ++k) u[k] += us[k];
        }
        const int qx = q % M, qy = (q / M) % M, qz = q / (M * M);
        const float wq = q < NQ ? Wt[qx] * Wt[qy] * Wt[qz] : 0.f;
        auto flux = [&]() {
            if (fhalf) tc_flux_half<P, 1>(u, q, ql, nel, meta(j), gamma, wq, sm + K::kG, status);
            else tc_flux_half<P, 0>(u, q, ql, nel, meta(j), gamma, wq, sm + K::kG, status);
        };
        auto gemm2 = [&](int ch) {
            // H[r][b] += sum_{q in chunk} G[r][q] B[q][b]: the operator read MN-major (b contiguous)
            constexpr uint32_t id2 = tc::idesc_bf16(128, NB, 1);
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const uint32_t ab = sbase + K::kG + tc::prod_a(s) * K::kGPart;
                const uint32_t bb = sbase + K::kOp + tc::prod_b(s) * K::kOpPart;
                const bool big = s == 5;
#pragma unroll
                for (int kl = 0; kl < K::KC / 16; ++kl)
                    tc::mma_bf16(big ? d2 : d2s, tc::sdesc(ab + kl * 32, 16, 1024),
                                 tc::sdesc(bb + (ch * (K::KC / 16) + kl) * 2048, K::kOpPart, 1024), id2,
                                 (ch > 0 || (big ? 0 : s) > 0 || kl > 0) ? 1u : 0u);
            }
            tc::mma_commit(bar2);
        };
        if (qt < 2) flux();
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            gemm2(0);
        }
        // ---- face lifts (FP32) while the first chunk multiplies (into the Uop region) ----
        for (int t2 = tid; t2 < E * 30; t2 += K::NT) {
            const int v = t2 % 5, f = (t2 / 5) % 6, e = t2 / 30;
            if (e >= nel) continue;
            const FaceRec& rec = r[e * 6 + f];
            const float* Fq = gF + (size_t)(rec.pad & 0x3fffffff) * FSTR + v * NF;
            const bool own = (rec.pad >> 30) & 1;
            const uint8_t* pm = a.cmap + (rec.info >> 4) * NF;
            float fl[NF];
#pragma unroll
            for (int c = 0; c < NF; ++c) fl[c] = __ldg(Fq + (own ? c : __ldg(pm + c)));
            const float sgn = ((rec.info >> 3) & 1) ? -1.f : 1.f;
            float tmp[M][N];
#pragma unroll
            for (int t1 = 0; t1 < M; ++t1)
#pragma unroll
                for (int b0 = 0; b0 < N; ++b0) {
                    float s = 0.f;
#pragma unroll
                    for (int t0 = 0; t0 < M; ++t0) s += Bt[t0 * N + b0] * fl[t1 * M + t0];
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
        // the first chunk has been read: the second overwrites it
        if (!(alive = wait_all(bar2, ph2))) break;
        ph2 ^= 1;
        tc::tc_fence_after();
        if (qt >= 2) flux();
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            gemm2(1);
        }
        if (!(alive = wait_all(bar2, ph2))) break;
        ph2 ^= 1;
        tc::tc_fence_after();
        // ---- Delta_d^T along each axis (FP32), one warp per direction and half ----
        {
            const int d = warp & 3, half = warp >> 2;
            if (d < 3) {
                const uint32_t lrow = static_cast<uint32_t>(d * 32) << 16;
                float h[32], hs[32];
                if (d < 2) {
                    tc::tmem_ld16(d2 + lrow + half * 32, h);
                    tc::tmem_ld16(d2 + lrow + half * 32 + 16, h + 16);
                    tc::tmem_ld16(d2s + lrow + half * 32, hs);
                    tc::tmem_ld16(d2s + lrow + half * 32 + 16, hs + 16);
                } else {
#pragma unroll
                    for (int bz = 0; bz < 4; ++bz) {
                        tc::tmem_ld8(d2 + lrow + bz * 16 + half * 8, h + bz * 8);
                        tc::tmem_ld8(d2s + lrow + bz * 16 + half * 8, hs + bz * 8);
                    }
                }
                tc::tmem_wait_ld();
#pragma unroll
                for (int k = 0; k < 32; ++k) h[k] += hs[k];
                const int c = lane;
                if (c < C && c / 5 < nel) {
                    float* out = Part + (d * C + c) * PS;
                    if (d == 0) {
                        // h[(bz - 2 half) * 16 + by * 4 + bx]
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj)
#pragma unroll
                            for (int bx = 0; bx < N; ++bx) {
                                float s = 0.f;
#pragma unroll
                                for (int i = 0; i < N; ++i) s += Dn[i * N + bx] * h[jj * 4 + i];
                                out[half * 32 + jj * 4 + bx] = s;
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
        // ---- residual (FP64): the three directions and the face lifts, summed in
        //      registers, then written over the partials ----
        constexpr int kPer = (C * NB + K::NT - 1) / K::NT;
        double rs[kPer];
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int i = tid + k * K::NT;
            rs[k] = 0.0;
            if (i >= C * NB) continue;
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
            rs[k] = s;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const int i = tid + k * K::NT;
            if (i < C * NB) Res[(i / NB) * PS + i % NB] = rs[k];
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
            const int c = i / N2, rr0 = i - c * N2;
            double* rr = Res + c * PS + rr0 * N;  // pencil along x at (by, bz)
            double t4[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t4[k] = rr[k];
#pragma unroll
            for (int jj = 0; jj < N; ++jj) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[jj * N + k] * t4[k];
                rr[jj] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < nel * 5 * N2; i += K::NT) {
            const int c = i / N2, rr0 = i - c * N2, bx = rr0 % N, bz = rr0 / N;
            double* rr = Res + c * PS + bz * N2 + bx;  // pencil along y
            double t4[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t4[k] = rr[k * N];
#pragma unroll
            for (int jj = 0; jj < N; ++jj) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[jj * N + k] * t4[k];
                rr[jj * N] = s;
            }
        }
        __syncthreads();
        for (int i = tid; i < nel * 5 * N2; i += K::NT) {
            const int c = i / N2, bxy = i - c * N2, e = c / 5;
            const GeoDev& gg = a.geo[cls(j)[e]];
            const double scale = a.dt * gg.dtf * gg.inv_djac;
            const double* rr = Res + c * PS + bxy;  // pencil along z
            double t4[N];
#pragma unroll
            for (int k = 0; k < N; ++k) t4[k] = rr[k * N2];
            const size_t gbase = (size_t)e0 * 5 * NB + (size_t)c * NB + bxy;
#pragma unroll
            for (int jj = 0; jj < N; ++jj) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < N; ++k) s += Mi[jj * N + k] * t4[k];
                const double kk = scale * s;
                const size_t gi = gbase + (size_t)jj * N2;
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
    // a CTA that stopped early may have record copies in flight: wait for them
    // (bounded) before the shared memory goes away
    if (tid == 0)
        for (int s2 = 0; s2 < 2; ++s2)
            if (pend[s2]) (void)tc::mbar_wait(barR0 + 8 * s2, pph[s2], kWait);
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
                   face_threads<P, float>(), launch_face_kernel<P, float, false>, face_batch<P, float>()};
    return v;
}

}  // namespace dgk
