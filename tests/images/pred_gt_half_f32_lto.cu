// count_if's `:pred` for x > 0.5 over floats (out = 1 or 0 as int), with its element function
// as LTO-IR so the runtime may fuse it with the '+' reduce of the ints.
#include "image_common.cuh"

extern "C" __device__ void parallax_elem(const void* in, void* out) {
    *static_cast<int*>(out) = *static_cast<const float*>(in) > 0.5f ? 1 : 0;
}

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const float* in = static_cast<const float*>(args.in);
    int* out = static_cast<int*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) parallax_elem(in + i, out + i);
}
