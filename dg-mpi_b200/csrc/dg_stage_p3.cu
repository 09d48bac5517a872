// dg_stage_p3.cu -- compiled launch variants of the stage kernel for order p = 3
// (elements per CTA, threads per CTA, variable groups, residual arithmetic; then the
// optional flags: all groups' pencils in one phase, single coefficient buffer, unfused
// volume, row-split traces and lifts, one face-flux point per thread, face fluxes from
// the face kernel, face lifts added in the inverse mass's first pass; then the minimum
// of resident CTAs per SM asked of the compiler).  Contexts on non-affine meshes use the
// general-geometry (kGE) entries only, the others never do.  The
// first variant of each precision is the default (the measured best); dg_tune_stage may pick another.
#include "dg_stage.cuh"
#include "dg_tc.cuh"

namespace dgk {

static const StageVariant kVariants3[] = {
    make_variant<3, 1, 96, 1, double, kUF | kSB | kFX | kMG>(),
    make_variant<3, 1, 128, 1, double, kUF | kSB | kFX | kMG>(),
    make_variant<3, 1, 128, 1, double, kUF | kRS | kSB | kFX | kMG>(),
    make_variant<3, 1, 128, 1, double, kUF | kSB | kFX>(),
    make_variant<3, 1, 128, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<3, 1, 128, 1, double, kUF | kRS | kSB | kFX, 8>(),
    make_variant<3, 1, 96, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<3, 1, 96, 1, double, kUF | kSB | kFX>(),
    make_variant<3, 1, 64, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<3, 2, 128, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<3, 1, 32, 1, double, kUF | kSB | kFX>(),
    make_variant<3, 1, 64, 1, double, kUF | kRS | kSB | kK1>(),
    make_variant<3, 1, 64, 1, double, kUF | kSB | kK1>(),
    make_variant<3, 1, 32, 2, double, kSB>(),
    make_variant<3, 2, 64, 2, double>(),
    make_variant<3, 1, 128, 1, float, kUF | kSB | kFX | kMG>(),
    make_variant<3, 1, 128, 1, float, kUF | kRS | kSB | kFX | kMG>(),
    make_variant<3, 1, 64, 1, float, kUF | kSB | kFX | kMG>(),
    make_variant<3, 1, 64, 1, float, kUF | kSB | kFX>(),
    make_variant<3, 1, 128, 1, float, kUF | kRS | kSB | kFX>(),
    make_variant<3, 1, 64, 1, float, kUF | kRS | kSB | kFX>(),
    make_variant<3, 1, 32, 1, float, kUF | kSB | kFX>(),
    make_variant<3, 1, 128, 1, float, kUF | kSB | kFX>(),
    make_variant<3, 1, 32, 1, float, kUF | kSB | kK1>(),
    make_variant<3, 1, 32, 1, float, kUF | kSB>(),
    make_variant<3, 2, 64, 1, float, kUF | kSB | kK1>(),
    make_variant<3, 1, 32, 1, float, kSB>(),
    make_variant<3, 1, 32, 1, float>(),
    // general (trilinear) geometry: the variants of non-affine meshes
    make_variant<3, 1, 64, 1, double, kUF | kRS | kSB | kK1 | kGE>(),
    make_variant<3, 1, 32, 1, float, kUF | kSB | kK1 | kGE>(),
    make_variant<3, 1, 64, 1, float, kUF | kSB | kK1 | kGE>(),
    make_variant<3, 1, 64, 1, float, kUF | kRS | kSB | kK1 | kGE>(),
    make_variant<3, 1, 128, 1, double, kUF | kRS | kSB | kGE | kFX>(),
    make_variant<3, 1, 128, 1, float, kUF | kSB | kGE | kFX>(),
    // the tensor-core kernel (split-TF32 volume integral)
    make_tc_variant<3>(),
};

int stage_variants_p3(const StageVariant** out)
{
    *out = kVariants3;
    return static_cast<int>(sizeof(kVariants3) / sizeof(kVariants3[0]));
}

}  // namespace dgk
