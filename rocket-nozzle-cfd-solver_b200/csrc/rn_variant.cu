// rn_variant.cu -- one precision variant of the time-step kernels.
//
// Compiled twice by the Makefile: -DRN_VARIANT=exact with IEEE division and
// square root, -DRN_VARIANT=fast with the hardware's approximate ones. Each
// compilation puts its kernels in namespace rn::<variant> and publishes them
// as rn::kernels_<variant> (see rn_kernels.cuh).
#ifndef RN_VARIANT
#error "RN_VARIANT must be defined (exact or fast)"
#endif
#include "rn_step.cu"
#include "rn_spray.cu"

#define RN_CAT_(a, b) a##b
#define RN_CAT(a, b) RN_CAT_(a, b)
#define RN_STR_(a) #a
#define RN_STR(a) RN_STR_(a)

namespace rn {
const KernelSet RN_CAT(kernels_, RN_VARIANT) = {
    RN_STR(RN_VARIANT),
    RN_VARIANT::launch_stage1,
    RN_VARIANT::launch_stage2,
    RN_VARIANT::launch_stage2phys,
    RN_VARIANT::launch_batch_stage1,
    RN_VARIANT::launch_batch_stage2,
    RN_VARIANT::launch_batch_stage2phys,
    RN_VARIANT::launch_reduce,
    RN_VARIANT::launch_rescale,
    RN_VARIANT::launch_wallrow,
    RN_VARIANT::launch_integrals,
    RN_VARIANT::launch_spray,
    RN_VARIANT::launch_apply,
    RN_VARIANT::spray_sort_temp_bytes,
    RN_VARIANT::stage_kernels_init,
};
}  // namespace rn
