// Run-time linking of registered images, and the fused transform + reduce.
//
// Reference: the transform_reduce and count_if funnels look up a transform kernel
// (":xform" / ":pred") and a '+' reduce (":reduce") and run them as two dispatches with a
// staging buffer between them (include/parallax/stdpar.hpp:245-293). When the transform's
// image also exports its per-element function as LTO-IR (parallax_elem, see
// include/parallax/kernel_abi.h), this file links it with the runtime's own reduce tile
// (csrc/lto/xform_reduce.cu, embedded in the library as LTO-IR) so that the pair runs as
// ONE pass over the input. nvJitLink inlines the element function into the tile.
//
// The same linker also loads images whose machine code is relocatable (compiled with
// -rdc), which the CUDA library loader may refuse: registry.cu links such an image alone.
#include <dlfcn.h>
#include <nvJitLink.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "runtime.hpp"

extern "C" const unsigned char pxb_lto_xform_reduce[];
extern "C" const size_t pxb_lto_xform_reduce_size;

namespace pxb {

namespace {

// nvJitLink, resolved at run time: the LTO-IR embedded here comes from the CUDA 12.9
// compiler and needs a 12.9 (or newer) linker, while a host program may already have loaded
// an older libnvJitLink.so.12 (Python frameworks bundle one). If the library the process
// resolves lacks the 12.9 entry points, the toolkit's copy is loaded into a namespace of its
// own (dlmopen), so both coexist.
struct JitLink {
    decltype(&__nvJitLinkCreate_12_9) create = nullptr;
    decltype(&__nvJitLinkAddData_12_9) add_data = nullptr;
    decltype(&__nvJitLinkComplete_12_9) complete = nullptr;
    decltype(&__nvJitLinkGetLinkedCubinSize_12_9) cubin_size = nullptr;
    decltype(&__nvJitLinkGetLinkedCubin_12_9) cubin = nullptr;
    decltype(&__nvJitLinkGetErrorLogSize_12_9) log_size = nullptr;
    decltype(&__nvJitLinkGetErrorLog_12_9) log = nullptr;
    decltype(&__nvJitLinkDestroy_12_9) destroy = nullptr;
    bool ok = false;

    bool resolve(void* lib) {
        if (!lib) return false;
        auto sym = [&](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(lib, name));
            return fn != nullptr;
        };
        return sym(create, "__nvJitLinkCreate_12_9") && sym(add_data, "__nvJitLinkAddData_12_9") &&
               sym(complete, "__nvJitLinkComplete_12_9") &&
               sym(cubin_size, "__nvJitLinkGetLinkedCubinSize_12_9") &&
               sym(cubin, "__nvJitLinkGetLinkedCubin_12_9") &&
               sym(log_size, "__nvJitLinkGetErrorLogSize_12_9") &&
               sym(log, "__nvJitLinkGetErrorLog_12_9") && sym(destroy, "__nvJitLinkDestroy_12_9");
    }
    JitLink() {
        if (resolve(dlopen("libnvJitLink.so.12", RTLD_NOW | RTLD_LOCAL))) {
            ok = true;
            return;
        }
        std::vector<std::string> dirs;
        for (const char* env : {"CUDA_HOME", "CUDA_PATH"})
            if (const char* d = getenv(env)) dirs.push_back(std::string(d) + "/lib64");
        dirs.push_back("/usr/local/cuda/lib64");
        for (const std::string& d : dirs) {
            const std::string path = d + "/libnvJitLink.so.12";
            if (resolve(dlmopen(LM_ID_NEWLM, path.c_str(), RTLD_NOW | RTLD_LOCAL))) {
                ok = true;
                return;
            }
        }
    }
};

const JitLink& jitlink() {
    static const JitLink api;
    return api;
}

}  // namespace

bool link_images(const std::vector<std::pair<const void*, size_t>>& inputs,
                 std::vector<char>* cubin, const char* what, bool quiet) {
    const JitLink& jl = jitlink();
    if (!jl.ok) {
        if (!quiet) set_error(PARALLAX_ERR_UNSUPPORTED, "%s: no nvJitLink 12.9 or newer", what);
        return false;
    }
    const char* opts[] = {"-arch=sm_100a", "-lto"};
    nvJitLinkHandle lh = nullptr;
    if (jl.create(&lh, 2, opts) != NVJITLINK_SUCCESS) {
        if (!quiet) set_error(PARALLAX_ERR_UNSUPPORTED, "%s: nvJitLinkCreate failed", what);
        return false;
    }
    bool ok = true;
    int idx = 0;
    for (const auto& in : inputs) {
        const std::string name = std::string(what) + "#" + std::to_string(idx++);
        if (jl.add_data(lh, NVJITLINK_INPUT_ANY, in.first, in.second, name.c_str()) !=
            NVJITLINK_SUCCESS) {
            ok = false;
            break;
        }
    }
    if (ok) ok = jl.complete(lh) == NVJITLINK_SUCCESS;
    size_t sz = 0;
    if (ok) ok = jl.cubin_size(lh, &sz) == NVJITLINK_SUCCESS && sz > 0;
    if (ok) {
        cubin->resize(sz);
        ok = jl.cubin(lh, cubin->data()) == NVJITLINK_SUCCESS;
    }
    if (!ok) {
        size_t log_size = 0;
        std::string log;
        if (jl.log_size(lh, &log_size) == NVJITLINK_SUCCESS && log_size > 1) {
            log.resize(log_size);
            jl.log(lh, &log[0]);
            log.resize(strnlen(log.c_str(), log.size()));
        }
        if (!quiet)
            set_error(PARALLAX_ERR_UNSUPPORTED, "%s: link failed%s%s", what,
                      log.empty() ? "" : ": ", log.substr(0, 300).c_str());
        else if (getenv("PARALLAX_DEBUG"))
            fprintf(stderr, "[parallax] %s: not linked%s%s\n", what, log.empty() ? "" : ": ",
                    log.substr(0, 300).c_str());
    }
    jl.destroy(&lh);
    return ok;
}

namespace {

std::mutex& fuse_mu() {
    static std::mutex m;
    return m;
}

const char* const kFusedNames[6] = {"pxb_xform_reduce_f32", "pxb_xform_reduce_f64",
                                    "pxb_xform_reduce_i32", "pxb_xform_reduce_i64",
                                    "pxb_xform_reduce_u32", "pxb_xform_reduce_u64"};

constexpr int kBlock = 256;
constexpr int kUnroll = 8;

}  // namespace

bool xform_fusable(Handle* h) {
    if (!h || h->kind != Kind::USER || h->image.empty()) return false;
    std::lock_guard<std::mutex> g(fuse_mu());
    if (h->fused_state) return h->fused_state == 1;
    h->fused_state = 2;
    // Linking fails (quietly: the two-pass path then runs) when the image has no LTO-IR
    // parallax_elem.
    std::vector<char> cubin;
    if (!link_images({{h->image.data(), h->image.size()},
                      {pxb_lto_xform_reduce, pxb_lto_xform_reduce_size}},
                     &cubin, "fused transform + reduce", true))
        return false;
    if (cudaLibraryLoadData(&h->fused_library, cubin.data(), nullptr, nullptr, 0, nullptr,
                            nullptr, 0) != cudaSuccess) {
        cudaGetLastError();
        h->fused_library = nullptr;
        return false;
    }
    for (int t = 0; t < 6; ++t) {
        if (cudaLibraryGetKernel(&h->fused[t], h->fused_library, kFusedNames[t]) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
    }
    h->fused_state = 1;
    return true;
}

bool launch_xform_reduce(Workspace& ws, Handle* xf, DType u, const void* d_in, size_t n,
                         size_t in_es, void* d_out) {
    const int t = (int)u;
    if (t < 0 || t >= 6 || xf->fused_state != 1) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "fused transform + reduce: unsupported type");
        return false;
    }
    char* scratch = ws.scratch(0);
    if (!scratch) return false;
    // accumulators are 8 bytes at most: the partials region holds this many
    constexpr size_t kMaxBlocks = (kScratchSmall - ScratchOff::partials) / 8;
    size_t blocks = (n + (size_t)kBlock * kUnroll - 1) / ((size_t)kBlock * kUnroll);
    const size_t cap = (size_t)device_info().sm_count * 8;
    if (blocks > cap) blocks = cap;
    if (blocks > kMaxBlocks) blocks = kMaxBlocks;
    if (blocks == 0) blocks = 1;
    const unsigned char* in = static_cast<const unsigned char*>(d_in);
    uint64_t count = n;
    uint32_t in_size = (uint32_t)in_es;
    void* partials = scratch + ScratchOff::partials;
    void* ticket = scratch + ScratchOff::ticket;
    void* args[] = {&in, &count, &in_size, &partials, &ticket, &d_out};
    count_launch();
    ProfScope prof(ws, "k_xform_reduce", (uint64_t)(n * in_es));
    return cuda_ok(cudaLaunchKernel((const void*)xf->fused[t], dim3((unsigned)blocks),
                                    dim3(kBlock), args, 0, ws.stream()),
                   "cudaLaunchKernel(fused transform + reduce)");
}

}  // namespace pxb
