/*
 * Launch convention for sm_100a images registered with parallax_kernel_register() or
 * loaded with parallax_kernel_load().
 *
 * The reference binds compiler-emitted SPIR-V to a fixed descriptor layout (in@0,
 * out@1, captures uniform@2, positions@3) and a 24-byte push block {count, host_base,
 * dev_base} (reference src/kernel/kernel_launcher.cpp:15-32, :188-204). The CUDA
 * equivalent is one kernel parameter block passed by value, so the captures live in
 * the kernel's constant parameter bank like a uniform buffer:
 *
 *     extern "C" __global__ void parallax_entry(parallax_launch_args args);
 *
 * The runtime launches `parallax_entry` with 256-thread blocks and a grid of at most
 * 148 * 16 blocks; the kernel must cover args.count elements with a grid-stride loop.
 * Stored host pointers into the arena are relocated in the kernel with
 *     device_address = args.dev_base + (host_pointer - args.host_base).
 *
 * Fusable transforms. A transform image registered under the key of a transform_reduce
 * (":xform") or count_if (":pred") funnel may also export its per-element function,
 *
 *     extern "C" __device__ void parallax_elem(const void* in, void* out);
 *
 * (reads one input element at `in`, writes the transformed element at `out`), as LTO-IR,
 * i.e. compiled relocatable with an LTO target beside the machine code:
 *
 *     nvcc -rdc=true -fatbin -gencode arch=compute_100a,code=[sm_100a,lto_100a] ...
 *
 * The runtime then links that function into its own reduce tile (nvJitLink, link-time
 * optimisation) and runs the funnel's transform2 + reduce pair as one pass over the input:
 * the transform2 call is held back until the reduce of its output, and any other call on
 * the same thread runs it first. An image without parallax_elem runs as two passes.
 */
#ifndef PARALLAX_KERNEL_ABI_H
#define PARALLAX_KERNEL_ABI_H

#define PARALLAX_MAX_CAPTURE_BYTES 256

typedef struct parallax_launch_args {
    void* in;                        /* element buffer (binding 0) */
    void* out;                       /* output buffer (binding 1); == in for in-place */
    unsigned long long count;        /* element count */
    unsigned long long in_elem_size;
    unsigned long long out_elem_size;
    unsigned long long host_base;    /* arena host mirror base */
    unsigned long long dev_base;     /* arena device base */
    unsigned long long capture_size;
    unsigned char captures[PARALLAX_MAX_CAPTURE_BYTES];  /* closure bytes (uniform@2) */
} parallax_launch_args;

#endif /* PARALLAX_KERNEL_ABI_H */
