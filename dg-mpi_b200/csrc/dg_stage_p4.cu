// dg_stage_p4.cu -- compiled launch variants of the stage kernel for order p = 4
// (elements per CTA, threads per CTA, variable groups, residual arithmetic; then the
// optional flags: all groups' pencils in one phase, single coefficient buffer).  The
// first variant of each precision is the default (the measured best); dg_tune_stage may pick another.
#include "dg_stage.cuh"

namespace dgk {

static const StageVariant kVariants4[] = {
    make_variant<4, 1, 64, 2, double>(),
    make_variant<4, 2, 96, 2, double>(),
    make_variant<4, 1, 128, 2, double>(),
    make_variant<4, 1, 32, 2, double>(),
    make_variant<4, 1, 32, 3, double>(),
    make_variant<4, 1, 64, 1, float>(),
    make_variant<4, 1, 128, 2, float, kPZ>(),
    make_variant<4, 1, 32, 2, float>(),
    make_variant<4, 1, 32, 1, float>(),
    make_variant<4, 2, 64, 1, float>(),
};

int stage_variants_p4(const StageVariant** out)
{
    *out = kVariants4;
    return static_cast<int>(sizeof(kVariants4) / sizeof(kVariants4[0]));
}

}  // namespace dgk
