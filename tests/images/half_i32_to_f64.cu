// transform: out[i] = (double)in[i] * 0.5, int -> double (different element sizes).
#include "image_common.cuh"

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const int* in = static_cast<const int*>(args.in);
    double* out = static_cast<double*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) out[i] = (double)in[i] * 0.5;
}
