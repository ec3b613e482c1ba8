// count_if's `:pred` transform for x > 0.5 over floats: out[i] = 1 or 0 as int
// (stdpar.hpp count_if funnel: transform float -> int, then a '+' reduce of the ints).
#include "image_common.cuh"

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const float* in = static_cast<const float*>(args.in);
    int* out = static_cast<int*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) out[i] = in[i] > 0.5f ? 1 : 0;
}
