// transform_reduce's `:xform` for long -> long, x * x (wrapping), element function as LTO-IR:
// an integer sum of the fused pass must equal the two-pass sum bit for bit.
#include "image_common.cuh"

extern "C" __device__ void parallax_elem(const void* in, void* out) {
    const unsigned long long x = (unsigned long long)*static_cast<const long long*>(in);
    *static_cast<long long*>(out) = (long long)(x * x);
}

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const long long* in = static_cast<const long long*>(args.in);
    long long* out = static_cast<long long*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) parallax_elem(in + i, out + i);
}
