// remove_if flags for the predicate x % 3 == 0 over int32: the elements to KEEP are those
// for which the predicate is false (one byte per element, 1 = keep).
#include "image_common.cuh"

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const int* in = static_cast<const int*>(args.in);
    uint8_t* flags = static_cast<uint8_t*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) flags[i] = in[i] % 3 != 0;
}
