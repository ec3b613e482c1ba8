// transform with captures over 16-byte records {float x; uint32 pad; float* p}:
// y[i] = a * x + *p, `a` the first 4 capture bytes, p a stored HOST pointer into the arena
// relocated in the kernel. Rounded multiply and add (bit-identical to host fp32).
#include "image_common.cuh"

struct Record { float x; uint32_t pad; const float* p; };

extern "C" __global__ void parallax_entry(parallax_launch_args args) {
    const float a = *reinterpret_cast<const float*>(args.captures);
    const Record* in = static_cast<const Record*>(args.in);
    float* out = static_cast<float*>(args.out);
    PARALLAX_FOR_EACH_INDEX(args, i) {
        const Record r = in[i];
        out[i] = __fadd_rn(__fmul_rn(a, r.x), *relocate(args, r.p));
    }
}
