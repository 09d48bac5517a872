// dg_stage_p5.cu -- compiled launch variants of the stage kernel for order p = 5
// (elements per CTA, threads per CTA, variable groups, residual arithmetic; then the
// optional flags: all groups' pencils in one phase, single coefficient buffer).  The
// first variant of each precision is the default (the measured best); dg_tune_stage may pick another.
#include "dg_stage.cuh"

namespace dgk {

static const StageVariant kVariants5[] = {
    make_variant<5, 1, 128, 3, double>(),
    make_variant<5, 1, 128, 3, double, kPZ>(),
    make_variant<5, 1, 64, 3, double>(),
    make_variant<5, 2, 128, 3, double>(),
    make_variant<5, 1, 32, 3, double>(),
    make_variant<5, 1, 128, 2, float, kSB>(),
    make_variant<5, 1, 128, 2, float>(),
    make_variant<5, 1, 64, 2, float>(),
    make_variant<5, 1, 64, 1, float>(),
    make_variant<5, 1, 32, 2, float>(),
    make_variant<5, 1, 32, 1, float>(),
};

int stage_variants_p5(const StageVariant** out)
{
    *out = kVariants5;
    return static_cast<int>(sizeof(kVariants5) / sizeof(kVariants5[0]));
}

}  // namespace dgk
