// dg_ensemble_f32.cu -- the ensemble launch kernels with the float residual
// (see dg_ensemble.cuh).
#include "dg_ensemble.cuh"

namespace dgk {

namespace {

size_t stage_smem_f32(unsigned mask)
{
    const size_t s[kMaxP + 1] = {0, ens_stage_smem<1, float>(), ens_stage_smem<2, float>(),
                                 ens_stage_smem<3, float>(), ens_stage_smem<4, float>(), ens_stage_smem<5, float>()};
    size_t m = 0;
    for (int p = 0; p <= kMaxP; ++p)
        if (mask & (1u << p)) m = s[p] > m ? s[p] : m;
    return m;
}

size_t face_smem_f32(unsigned mask)
{
    const size_t s[kMaxP + 1] = {0, face_smem_bytes<1, float>(), face_smem_bytes<2, float>(), face_smem_bytes<3, float>(),
                                 face_smem_bytes<4, float>(), face_smem_bytes<5, float>()};
    size_t m = 0;
    for (int p = 0; p <= kMaxP; ++p)
        if (mask & (1u << p)) m = s[p] > m ? s[p] : m;
    return m;
}

cudaError_t launch_stage_f32(const EnsembleArgs& a, int grid, size_t smem, cudaStream_t s)
{
    ensemble_stage_kernel<float><<<grid, kEnsThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_face_f32(const EnsembleArgs& a, int grid, size_t smem, cudaStream_t s)
{
    ensemble_face_kernel<float><<<grid, kFaceThreads, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

EnsembleKernels ensemble_kernels_f32()
{
    return EnsembleKernels{(const void*)ensemble_stage_kernel<float>, (const void*)ensemble_face_kernel<float>,
                           stage_smem_f32, face_smem_f32, launch_stage_f32, launch_face_f32};
}

}  // namespace dgk
