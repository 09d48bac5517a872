// dg_ensemble.cuh -- one launch per RK stage for an ensemble of cases of
// different orders: the stage kernel (and, before it, the face-flux kernel)
// of every order group in a single grid.
//
// The blocks of the grid are split into one range per group, in proportion to
// the group's work, as the starting point: a block runs its group's stage
// body (stage_body of its order, 128 threads per block for every order),
// claiming the group's element batches from the group's work counter, and
// when those run out it moves on to the other groups' batches -- so the
// launch ends when all work is done, whatever the split.  The per-order
// launch configurations below
// are compiled launch variants of the orders (128 threads per CTA), so a
// single context running the same variant computes bit for bit what the
// ensemble launch computes for it.  Dynamic shared memory is that of the
// largest order present.
#pragma once
#include "dg_stage.cuh"

namespace dgk {

constexpr int kEnsThreads = 128;
constexpr int kEnsMaxGroups = kMaxP + 1;
// orders 1..5 (p = 0 groups keep their own launches); resident CTAs per SM
// asked of the compiler: the register cap of the largest order's body
constexpr unsigned kEnsOrders = 0x3Eu;
template <typename T> struct EnsMinBlocks { static constexpr int value = sizeof(T) == 4 ? 4 : 2; };
// the same for the face kernels (the largest order's face body: 72 / 140 registers)
template <typename T> struct EnsFaceMinBlocks { static constexpr int value = sizeof(T) == 4 ? 6 : 3; };

struct EnsembleArgs {
    int ngroup;
    int order[kEnsMaxGroups];
    int blk[kEnsMaxGroups + 1];   // group g's blocks start in [blk[g], blk[g+1])
    int* work;                    // [ngroup] batch counters of this launch, zero before it
    StageArgs g[kEnsMaxGroups];
};

// the launch configuration of order P in an ensemble launch: elements per
// CTA and launch options (128 threads, one variable group)
template <int P, bool F32>
struct EnsCfg;
template <bool F32> struct EnsCfg<0, F32> { static constexpr int E = 32, FL = 0; };
template <> struct EnsCfg<1, true> { static constexpr int E = 8, FL = kUF | kSB | kFX; };
template <> struct EnsCfg<1, false> { static constexpr int E = 8, FL = 0; };
template <bool F32> struct EnsCfg<2, F32> { static constexpr int E = 4, FL = kUF | kSB | kFX; };
template <bool F32> struct EnsCfg<3, F32> { static constexpr int E = 1, FL = kUF | kSB | kFX; };
template <bool F32> struct EnsCfg<4, F32> { static constexpr int E = 1, FL = kUF | kSB | kFX; };
template <bool F32> struct EnsCfg<5, F32> { static constexpr int E = 1, FL = kUF | kRS | kSB | kFX; };

// host: the configuration of order p as (E, launch options)
inline void ensemble_config(int p, bool fp32, int& E, int& flags)
{
    switch (p) {
        case 0: E = EnsCfg<0, true>::E; flags = EnsCfg<0, true>::FL; break;
        case 1: E = fp32 ? EnsCfg<1, true>::E : EnsCfg<1, false>::E; flags = fp32 ? EnsCfg<1, true>::FL : EnsCfg<1, false>::FL; break;
        case 2: E = EnsCfg<2, true>::E; flags = EnsCfg<2, true>::FL; break;
        case 3: E = EnsCfg<3, true>::E; flags = EnsCfg<3, true>::FL; break;
        case 4: E = EnsCfg<4, true>::E; flags = EnsCfg<4, true>::FL; break;
        default: E = EnsCfg<5, true>::E; flags = EnsCfg<5, true>::FL; break;
    }
}

template <int P, typename T>
constexpr size_t ens_stage_smem()
{
    using C = EnsCfg<P, sizeof(T) == 4>;
    return stage_smem_bytes<P, C::E, 1, T, C::FL>();
}

// which group a block belongs to, and its index / count within the group
__device__ __forceinline__ int ens_group(const EnsembleArgs& a, int& bid, int& nblk)
{
    int g = 0;
    while (g + 1 < a.ngroup && (int)blockIdx.x >= a.blk[g + 1]) ++g;
    bid = (int)blockIdx.x - a.blk[g];
    nblk = a.blk[g + 1] - a.blk[g];
    return g;
}

template <typename T>
__global__ void __launch_bounds__(kEnsThreads, EnsMinBlocks<T>::value) ensemble_stage_kernel(const __grid_constant__ EnsembleArgs a)
{
    constexpr bool F = sizeof(T) == 4;
    __shared__ int slots[2];
    int bid, nblk;
    const int g0 = ens_group(a, bid, nblk);
    for (int t = 0; t < a.ngroup; ++t) {
        const int g = g0 + t < a.ngroup ? g0 + t : g0 + t - a.ngroup;
        const StageArgs& s = a.g[g];
        int* w = a.work + g;
        switch (a.order[g]) {
            case 1: stage_body<1, EnsCfg<1, F>::E, kEnsThreads, 1, T, EnsCfg<1, F>::FL>(s, 0, 1, w, slots); break;
            case 2: stage_body<2, EnsCfg<2, F>::E, kEnsThreads, 1, T, EnsCfg<2, F>::FL>(s, 0, 1, w, slots); break;
            case 3: stage_body<3, EnsCfg<3, F>::E, kEnsThreads, 1, T, EnsCfg<3, F>::FL>(s, 0, 1, w, slots); break;
            case 4: stage_body<4, EnsCfg<4, F>::E, kEnsThreads, 1, T, EnsCfg<4, F>::FL>(s, 0, 1, w, slots); break;
            default: stage_body<5, EnsCfg<5, F>::E, kEnsThreads, 1, T, EnsCfg<5, F>::FL>(s, 0, 1, w, slots); break;
        }
        __syncthreads();  // shared memory is reused by the next group's body
    }
}

// the face-flux kernels of the groups whose configuration has the face kernel
// (kFaceThreads = 128 threads per block for every order)
template <typename T>
__global__ void __launch_bounds__(kFaceThreads, EnsFaceMinBlocks<T>::value) ensemble_face_kernel(const __grid_constant__ EnsembleArgs a)
{
    __shared__ int slots[2];
    int bid, nblk;
    const int g0 = ens_group(a, bid, nblk);
    for (int t = 0; t < a.ngroup; ++t) {
        const int g = g0 + t < a.ngroup ? g0 + t : g0 + t - a.ngroup;
        const StageArgs& s = a.g[g];
        if (s.nface <= s.face_begin) continue;  // no face kernel in this group's configuration
        int* w = a.work + g;
        switch (a.order[g]) {
            case 1: face_flux_body<1, T, false>(s, 0, 1, w, slots); break;
            case 2: face_flux_body<2, T, false>(s, 0, 1, w, slots); break;
            case 3: face_flux_body<3, T, false>(s, 0, 1, w, slots); break;
            case 4: face_flux_body<4, T, false>(s, 0, 1, w, slots); break;
            case 5: face_flux_body<5, T, false>(s, 0, 1, w, slots); break;
            default: break;
        }
        __syncthreads();
    }
}

// host side (dg_ensemble_f32.cu / dg_ensemble_f64.cu): dynamic shared memory
// of the two kernels for the orders present (mask bit p), the kernels for
// attributes and occupancy, and the launches
struct EnsembleKernels {
    const void* stage;
    const void* face;
    size_t (*stage_smem)(unsigned order_mask);
    size_t (*face_smem)(unsigned order_mask);
    cudaError_t (*launch_stage)(const EnsembleArgs&, int grid, size_t smem, cudaStream_t);
    cudaError_t (*launch_face)(const EnsembleArgs&, int grid, size_t smem, cudaStream_t);
};
EnsembleKernels ensemble_kernels_f32();
EnsembleKernels ensemble_kernels_f64();
inline EnsembleKernels ensemble_kernels(bool fp32) { return fp32 ? ensemble_kernels_f32() : ensemble_kernels_f64(); }

}  // namespace dgk
