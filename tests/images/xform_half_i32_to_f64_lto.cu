// transform_reduce's `:xform` for int -> double, x * 0.5, with its element function as LTO-IR
// (built relocatable with an lto_100a target; see kernel_abi.h), so the runtime may fuse it
// with the reduce that follows.
#include "image_common.cuh"

extern "C" __device__ void parallax_elem(const void* in, void* out) {
    *static_cast<double*>(out) = (double)*static_cast<const int*>(in) * 0.5;
}

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const int* in = static_cast<const int*>(args.in);
    double* out = static_cast<double*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) parallax_elem(in + i, out + i);
}
