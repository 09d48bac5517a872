// dg_ensemble_f64.cu -- the ensemble launch kernels with the double residual
// (see dg_ensemble.cuh).
#include "dg_ensemble.cuh"

namespace dgk {

namespace {

size_t stage_smem_f64(unsigned mask)
{
    const size_t s[kMaxP + 1] = {0, ens_stage_smem<1, double>(), ens_stage_smem<2, double>(),
                                 ens_stage_smem<3, double>(), ens_stage_smem<4, double>(), ens_stage_smem<5, double>()};
    size_t m = 0;
    for (int p = 0; p <= kMaxP; ++p)
        if (mask & (1u << p)) m = s[p] > m ? s[p] : m;
    return m;
}

size_t face_smem_f64(unsigned mask)
{
    const size_t s[kMaxP + 1] = {0, face_smem_bytes<1, double>(), face_smem_bytes<2, double>(), face_smem_bytes<3, double>(),
                                 face_smem_bytes<4, double>(), face_smem_bytes<5, double>()};
    size_t m = 0;
    for (int p = 0; p <= kMaxP; ++p)
        if (mask & (1u << p)) m = s[p] > m ? s[p] : m;
    return m;
}

cudaError_t launch_stage_f64(const EnsembleArgs& a, int grid, size_t smem, cudaStream_t s)
{
    ensemble_stage_kernel<double><<<grid, kEnsThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_face_f64(const EnsembleArgs& a, int grid, size_t smem, cudaStream_t s)
{
    ensemble_face_kernel<double><<<grid, kFaceThreads, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

EnsembleKernels ensemble_kernels_f64()
{
    return EnsembleKernels{(const void*)ensemble_stage_kernel<double>, (const void*)ensemble_face_kernel<double>,
                           stage_smem_f64, face_smem_f64, launch_stage_f64, launch_face_f64};
}

}  // namespace dgk
