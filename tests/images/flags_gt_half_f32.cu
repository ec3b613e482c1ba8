// copy_if flags for x > 0.5 over floats: the predicate of the reference's own flags shader
// (shaders/flags.comp:14-18), one byte per element instead of a float 1.0 / 0.0.
#include "image_common.cuh"

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const float* in = static_cast<const float*>(args.in);
    uint8_t* flags = static_cast<uint8_t*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) flags[i] = in[i] > 0.5f;
}
