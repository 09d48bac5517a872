// dg_stage_p5.cu -- compiled launch variants of the stage kernel for order p = 5
// (elements per CTA, threads per CTA, variable groups); the first entry is
// the default, the tuner (dg_tune_stage) may pick another.
#include "dg_stage.cuh"

namespace dgk {

static const StageVariant kVariants5[] = {
    make_variant<5, 1, 32, 3>(),
    make_variant<5, 2, 128, 3>(),
    make_variant<5, 1, 64, 3>(),
    make_variant<5, 2, 64, 3>(),
};

int stage_variants_p5(const StageVariant** out)
{
    *out = kVariants5;
    return static_cast<int>(sizeof(kVariants5) / sizeof(kVariants5[0]));
}

}  // namespace dgk
