// dg_stage_p5.cu -- compiled launch variants of the stage kernel for order p = 5
// (elements per CTA, threads per CTA, variable groups, residual arithmetic; then the
// optional flags: all groups' pencils in one phase, single coefficient buffer, unfused
// volume, row-split traces and lifts, one face-flux point per thread, face fluxes from
// the face kernel, face lifts added in the inverse mass's first pass; then the minimum
// of resident CTAs per SM asked of the compiler).  Contexts on non-affine meshes use the
// general-geometry (kGE) entries only, the others never do.  The
// first variant of each precision is the default (the measured best); dg_tune_stage may pick another.
#include "dg_stage.cuh"

namespace dgk {

static const StageVariant kVariants5[] = {
    make_variant<5, 1, 256, 1, double, kUF | kRS | kSB | kFX | kMG, 2>(),
    make_variant<5, 1, 192, 1, double, kUF | kRS | kSB | kFX | kMG>(),
    make_variant<5, 1, 256, 1, double, kUF | kRS | kSB | kFX, 2>(),
    make_variant<5, 1, 192, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<5, 1, 128, 1, double, kUF | kRS | kSB | kFX>(),
    make_variant<5, 1, 256, 1, double, kUF | kRS | kSB | kK1, 2>(),
    make_variant<5, 1, 128, 1, double, kUF | kRS | kSB | kK1>(),
    make_variant<5, 1, 128, 3, double>(),
    make_variant<5, 1, 256, 1, float, kUF | kSB | kFX | kMG, 3>(),
    make_variant<5, 1, 256, 1, float, kUF | kRS | kSB | kFX | kMG, 3>(),
    make_variant<5, 1, 256, 1, float, kUF | kRS | kSB | kFX, 3>(),
    make_variant<5, 1, 128, 1, float, kUF | kRS | kSB | kFX>(),
    make_variant<5, 1, 256, 1, float, kUF | kSB | kFX, 3>(),
    make_variant<5, 1, 256, 1, float, kUF | kRS | kSB | kK1, 3>(),
    make_variant<5, 1, 128, 1, float, kUF | kRS | kSB | kK1>(),
    make_variant<5, 1, 128, 2, float, kSB>(),
    make_variant<5, 1, 64, 2, float>(),
    // general (trilinear) geometry: the variants of non-affine meshes
    make_variant<5, 1, 256, 1, double, kUF | kRS | kSB | kK1 | kGE, 2>(),
    make_variant<5, 1, 128, 1, float, kUF | kRS | kSB | kK1 | kGE>(),
    make_variant<5, 1, 128, 1, double, kUF | kRS | kSB | kK1 | kGE>(),
    make_variant<5, 1, 256, 1, float, kUF | kRS | kSB | kK1 | kGE, 3>(),
    make_variant<5, 1, 256, 1, double, kUF | kRS | kSB | kGE | kFX, 2>(),
    make_variant<5, 1, 256, 1, float, kUF | kRS | kSB | kGE | kFX, 3>(),
};

int stage_variants_p5(const StageVariant** out)
{
    *out = kVariants5;
    return static_cast<int>(sizeof(kVariants5) / sizeof(kVariants5[0]));
}

}  // namespace dgk
