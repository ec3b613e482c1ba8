// for_each over 8-byte records {float* p}: *p += 1 through a stored HOST pointer into the
// arena (a kernel that writes memory other than its operand).
#include "image_common.cuh"

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    float* const* in = static_cast<float* const*>(args.in);
    PARALLAX_FOR_EACH_INDEX(args, i) {
        float* p = relocate(args, in[i]);
        *p = *p + 1.0f;
    }
}
