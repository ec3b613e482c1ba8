// copy_if / partition flags for the predicate "x is odd" over int64 (8-byte elements).
#include "image_common.cuh"

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const long long* in = static_cast<const long long*>(args.in);
    uint8_t* flags = static_cast<uint8_t*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) flags[i] = (in[i] & 1) != 0;
}
