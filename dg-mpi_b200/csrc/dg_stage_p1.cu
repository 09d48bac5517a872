// dg_stage_p1.cu -- compiled launch variants of the stage kernel for order p = 1
// (elements per CTA, threads per CTA, variable groups, residual arithmetic; then the
// optional flags: all groups' pencils in one phase, single coefficient buffer, unfused
// volume, row-split traces and lifts, one face-flux point per thread, face fluxes from
// the face kernel, face lifts added in the inverse mass's first pass; then the minimum
// of resident CTAs per SM asked of the compiler).  Contexts on non-affine meshes use the
// general-geometry (kGE) entries only, the others never do.  The
// first variant of each precision is the default (the measured best); dg_tune_stage may pick another.
#include "dg_stage.cuh"

namespace dgk {

static const StageVariant kVariants1[] = {
    make_variant<1, 8, 128, 1, double>(),
    make_variant<1, 4, 64, 1, double>(),
    make_variant<1, 2, 64, 1, double>(),
    make_variant<1, 1, 32, 1, double>(),
    make_variant<1, 8, 128, 1, float, kUF | kSB | kFX>(),
    make_variant<1, 4, 64, 1, float, kUF | kSB | kFX>(),
    make_variant<1, 8, 128, 1, float>(),
    make_variant<1, 4, 64, 1, float>(),
    make_variant<1, 2, 64, 1, float>(),
    // general (trilinear) geometry: the variants of non-affine meshes
    make_variant<1, 2, 64, 1, double, kUF | kGE>(),
    make_variant<1, 2, 64, 1, float, kUF | kGE>(),
};

int stage_variants_p1(const StageVariant** out)
{
    *out = kVariants1;
    return static_cast<int>(sizeof(kVariants1) / sizeof(kVariants1[0]));
}

}  // namespace dgk
