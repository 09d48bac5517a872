// dg_stage_p2.cu -- compiled launch variants of the stage kernel for order p = 2
// (elements per CTA, threads per CTA, variable groups, residual arithmetic; then the
// optional flags: all groups' pencils in one phase, single coefficient buffer, unfused
// volume, row-split traces and lifts, one face-flux point per thread, face fluxes from
// the face kernel, face lifts added in the inverse mass's first pass; then the minimum
// of resident CTAs per SM asked of the compiler).  Contexts on non-affine meshes use the
// general-geometry (kGE) entries only, the others never do.  The
// first variant of each precision is the default (the measured best); dg_tune_stage may pick another.
#include "dg_stage.cuh"

namespace dgk {

static const StageVariant kVariants2[] = {
    make_variant<2, 1, 32, 1, double, kUF | kSB | kFX | kMG>(),
    make_variant<2, 2, 64, 1, double, kUF | kSB | kFX | kMG>(),
    make_variant<2, 1, 32, 1, double, kUF | kSB | kFX>(),
    make_variant<2, 2, 64, 1, double, kUF | kSB | kFX>(),
    make_variant<2, 1, 64, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<2, 1, 32, 1, double, kUF>(),
    make_variant<2, 2, 64, 1, double, kUF | kRS | kSB>(),
    make_variant<2, 1, 32, 1, double>(),
    make_variant<2, 2, 64, 1, double>(),
    make_variant<2, 1, 32, 1, float, kUF | kSB | kFX | kMG>(),
    make_variant<2, 2, 64, 1, float, kUF | kSB | kFX | kMG>(),
    make_variant<2, 1, 32, 1, float, kUF | kSB | kFX>(),
    make_variant<2, 2, 64, 1, float, kUF | kSB | kFX>(),
    make_variant<2, 1, 64, 1, float, kUF | kRS | kSB | kFX>(),
    make_variant<2, 1, 32, 1, float, kUF>(),
    make_variant<2, 2, 64, 1, float, kUF | kSB>(),
    make_variant<2, 4, 128, 1, float>(),
    make_variant<2, 1, 32, 1, float>(),
    // general (trilinear) geometry: the variants of non-affine meshes
    make_variant<2, 1, 32, 1, double, kUF | kGE>(),
    make_variant<2, 1, 32, 1, float, kUF | kGE>(),
    make_variant<2, 1, 32, 1, double, kUF | kSB | kGE | kFX>(),
    make_variant<2, 1, 32, 1, float, kUF | kSB | kGE | kFX>(),
    // 128 threads per CTA (the ensemble launch's block size for every order)
    make_variant<2, 4, 128, 1, double, kUF | kSB | kFX>(),
    make_variant<2, 4, 128, 1, float, kUF | kSB | kFX>(),
};

int stage_variants_p2(const StageVariant** out)
{
    *out = kVariants2;
    return static_cast<int>(sizeof(kVariants2) / sizeof(kVariants2[0]));
}

}  // namespace dgk
