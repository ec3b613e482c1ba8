// String-keyed kernel registry and kernel handles.
//
// Replaces the reference registry (src/kernel/cache.cpp:39-104) and pipeline loader
// (src/kernel/kernel_launcher.cpp:160-275). The reference stores SPIR-V and builds a
// Vulkan pipeline on first lookup. Here a handle is one of:
//   * a built-in sm_100a primitive (reduce / scan / sort / compaction / search / map),
//     selected by parsing the funnel key the stdpar header builds from
//     __PRETTY_FUNCTION__ (e.g. "T parallax::detail::device_reduce(const T*, ...)
//     [with T = float; ...]", suffixed ":scan", ":add", ":shift", ":flags", ":scatter"),
//     or by an explicit spec string (parallax_builtin_kernel);
//   * a registered / loaded sm_100a cubin or fatbin, loaded lazily through the CUDA
//     library API and launched through the parallax_entry convention (kernel_abi.h).
// A registered SPIR-V image cannot run here; its key still resolves when it names a
// fixed primitive funnel (those shaders are the reference's generic kernels), and
// misses otherwise, which sends the caller to its host loop exactly as a reference
// lookup miss does. The registry is guarded by a mutex (the reference's map is not).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cctype>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace pxb {

namespace {

struct Entry {
    const unsigned int* image = nullptr;
    size_t words = 0;
    Handle* handle = nullptr;
    bool resolved = false;
};

std::mutex& reg_mu() {
    static std::mutex* m = new std::mutex();
    return *m;
}
std::map<std::string, Entry>& registry() {
    static auto* r = new std::map<std::string, Entry>();
    return *r;
}
// Handles are owned by the runtime and never freed (as in the reference,
// src/kernel/cache.cpp:61); built-in handles are interned by spec.
std::map<std::string, Handle*>& interned() {
    static auto* m = new std::map<std::string, Handle*>();
    return *m;
}

bool debug() {
    static const bool on = getenv("PARALLAX_DEBUG") != nullptr;
    return on;
}

constexpr uint32_t kSpirvMagic = 0x07230203u;
constexpr uint32_t kElfMagic = 0x464c457fu;      // "\x7fELF" little endian
constexpr uint32_t kFatbinMagic = 0xba55ed50u;   // fatbin container header

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && isspace((unsigned char)s[a])) ++a;
    while (b > a && isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

DType dtype_from_cxx(std::string t) {
    t = trim(t);
    // strip cv-qualifiers the pretty printer may keep
    for (const char* q : {"const ", "volatile "})
        while (t.compare(0, strlen(q), q) == 0) t = t.substr(strlen(q));
    static const std::map<std::string, DType> names = {
        {"float", DType::F32},
        {"double", DType::F64},
        {"int", DType::I32},
        {"signed int", DType::I32},
        {"int32_t", DType::I32},
        {"std::int32_t", DType::I32},
        {"unsigned int", DType::U32},
        {"unsigned", DType::U32},
        {"uint32_t", DType::U32},
        {"std::uint32_t", DType::U32},
        {"long", DType::I64},
        {"long int", DType::I64},
        {"long long", DType::I64},
        {"long long int", DType::I64},
        {"int64_t", DType::I64},
        {"std::int64_t", DType::I64},
        {"unsigned long", DType::U64},
        {"long unsigned int", DType::U64},
        {"unsigned long long", DType::U64},
        {"long long unsigned int", DType::U64},
        {"uint64_t", DType::U64},
        {"std::uint64_t", DType::U64},
        {"std::size_t", DType::U64},
        {"size_t", DType::U64},
    };
    auto it = names.find(t);
    return it == names.end() ? DType::INVALID : it->second;
}

DType dtype_from_spec(const std::string& s) {
    static const std::map<std::string, DType> names = {
        {"f32", DType::F32}, {"f64", DType::F64}, {"i32", DType::I32},
        {"i64", DType::I64}, {"u32", DType::U32}, {"u64", DType::U64}};
    auto it = names.find(s);
    return it == names.end() ? DType::INVALID : it->second;
}

// Value of the template parameter `name` in a pretty-function string:
// GCC "[with T = float; std::size_t = ...]", Clang "[T = float]".
std::string template_arg(const std::string& key, const std::string& name) {
    size_t lb = key.rfind('[');
    if (lb == std::string::npos) return "";
    std::string pat = name + " = ";
    size_t p = key.find(pat, lb);
    while (p != std::string::npos && p > 0 && (isalnum((unsigned char)key[p - 1]) ||
                                               key[p - 1] == '_' || key[p - 1] == ':'))
        p = key.find(pat, p + 1);
    if (p == std::string::npos) return "";
    p += pat.size();
    size_t e = p;
    int depth = 0;
    while (e < key.size()) {
        char c = key[e];
        if (c == '<' || c == '(') ++depth;
        if (c == '>' || c == ')') --depth;
        if (depth == 0 && (c == ';' || c == ']' || c == ',')) break;
        ++e;
    }
    return trim(key.substr(p, e - p));
}

Handle* intern(const std::string& spec, const Handle& proto) {
    auto& m = interned();
    auto it = m.find(spec);
    if (it != m.end()) return it->second;
    Handle* h = new Handle(proto);
    h->name = spec;
    m[spec] = h;
    return h;
}

// Built-in handle for a fixed primitive funnel key, or nullptr.
Handle* funnel_builtin(const std::string& key) {
    size_t p = key.find("device_");
    if (p == std::string::npos) return nullptr;
    size_t e = p + 7;
    while (e < key.size() && (isalnum((unsigned char)key[e]) || key[e] == '_')) ++e;
    std::string funnel = key.substr(p + 7, e - p - 7);
    std::string suffix;
    size_t colon = key.rfind(':');
    size_t rb = key.rfind(']');
    if (colon != std::string::npos && rb != std::string::npos && colon > rb)
        suffix = key.substr(colon + 1);
    DType t = dtype_from_cxx(template_arg(key, "T"));
    if (t == DType::INVALID) return nullptr;
    Handle proto;
    proto.dtype = t;
    std::string dt = std::to_string((int)t);
    if (funnel == "reduce" && suffix.empty()) {
        proto.kind = Kind::REDUCE;
        proto.op = RedOp::SUM;
        return intern("funnel:reduce:" + dt, proto);
    }
    if (funnel == "scan" || funnel == "exclusive_scan") {
        if (suffix == "scan") proto.kind = Kind::SCAN;
        else if (suffix == "add") proto.kind = Kind::SCAN_ADD;
        else if (suffix == "shift" && funnel == "exclusive_scan") proto.kind = Kind::EXSCAN_SHIFT;
        else return nullptr;
        return intern("funnel:" + funnel + ":" + suffix + ":" + dt, proto);
    }
    if (funnel == "sort" && suffix.empty()) {
        proto.kind = Kind::SORT;
        return intern("funnel:sort:" + dt, proto);
    }
    if (funnel == "unique") {
        if (suffix == "flags") proto.kind = Kind::UNIQUE_FLAGS;
        else if (suffix == "scan") proto.kind = Kind::SCAN;
        else if (suffix == "add") proto.kind = Kind::SCAN_ADD;
        else if (suffix == "scatter") proto.kind = Kind::COMPACT_SCATTER;
        else return nullptr;
        return intern("funnel:unique:" + suffix + ":" + dt, proto);
    }
    // copy_if / remove_if / partition carry a user predicate: their `:flags` kernel must be
    // a registered sm_100a image (parallax_copy_if runs it, then the built-in compaction).
    // The other three keys of these funnels name generic kernels (scan of the flags, add,
    // scatter) and resolve to built-in handles, so a compiler registers only `:flags`.
    if (funnel == "copy_if" || funnel == "remove_if" || funnel == "partition") {
        if (suffix == "scan") proto.kind = Kind::SCAN;
        else if (suffix == "add") proto.kind = Kind::SCAN_ADD;
        else if (suffix == "scatter")
            proto.kind = funnel == "partition" ? Kind::PARTITION_SCATTER : Kind::COMPACT_SCATTER;
        else return nullptr;
        return intern("funnel:" + funnel + ":" + suffix + ":" + dt, proto);
    }
    // count_if / transform_reduce: the `:pred` / `:xform` transform is a registered image;
    // the `:reduce` kernel is the built-in '+' reduce of the transform's result type (int
    // for count_if, stdpar.hpp:271-293; U for transform_reduce, stdpar.hpp:245-267).
    if ((funnel == "count_if" || funnel == "transform_reduce") && suffix == "reduce") {
        const DType r = funnel == "count_if" ? DType::I32 : dtype_from_cxx(template_arg(key, "U"));
        if (r == DType::INVALID) return nullptr;
        proto.kind = Kind::REDUCE;
        proto.op = RedOp::SUM;
        proto.dtype = r;
        return intern("funnel:" + funnel + ":reduce:" + std::to_string((int)r), proto);
    }
    // transform / invoke and the `:flags`, `:pred`, `:xform` kernels carry a user functor:
    // they need a registered sm_100a image.
    return nullptr;
}

bool parse_number(const std::string& s, double* f, int64_t* i, uint64_t* u) {
    if (s.empty()) return false;
    char* end = nullptr;
    *f = strtod(s.c_str(), &end);
    if (*end) return false;
    *i = strtoll(s.c_str(), &end, 0);
    if (*end) *i = (int64_t)*f;
    *u = strtoull(s.c_str(), &end, 0);
    if (*end || s[0] == '-') *u = (uint64_t)*i;
    return true;
}

std::vector<std::string> split(const std::string& s, char c) {
    std::vector<std::string> out;
    size_t a = 0;
    for (;;) {
        size_t b = s.find(c, a);
        out.push_back(s.substr(a, b == std::string::npos ? std::string::npos : b - a));
        if (b == std::string::npos) break;
        a = b + 1;
    }
    return out;
}

bool parse_pred(const std::vector<std::string>& f, size_t at, Pred* p) {
    if (at >= f.size()) return false;
    const std::string& k = f[at];
    static const std::map<std::string, PredKind> kinds = {
        {"gt", PredKind::GT}, {"ge", PredKind::GE}, {"lt", PredKind::LT},
        {"le", PredKind::LE}, {"eq", PredKind::EQ}, {"ne", PredKind::NE},
        {"mod", PredKind::MOD}, {"nonzero", PredKind::NONZERO}};
    auto it = kinds.find(k);
    if (it == kinds.end()) return false;
    p->kind = it->second;
    if (p->kind == PredKind::NONZERO) return at + 1 == f.size();
    if (p->kind == PredKind::MOD) {
        if (at + 3 != f.size()) return false;
        double fd;
        int64_t m, r;
        uint64_t u;
        if (!parse_number(f[at + 1], &fd, &m, &u) || !parse_number(f[at + 2], &fd, &r, &u))
            return false;
        if (m == 0) return false;
        p->mod_m = m;
        p->mod_r = r;
        return true;
    }
    if (at + 2 != f.size()) return false;
    return parse_number(f[at + 1], &p->f, &p->i, &p->u);
}

Handle* parse_spec(const std::string& spec) {
    auto f = split(spec, ':');
    if (f.empty()) return nullptr;
    Handle h;
    const std::string& op = f[0];
    if (op == "reduce") {
        if (f.size() != 3) return nullptr;
        h.kind = Kind::REDUCE;
        if (f[1] == "sum") h.op = RedOp::SUM;
        else if (f[1] == "max") h.op = RedOp::MAX;
        else if (f[1] == "min") h.op = RedOp::MIN;
        else return nullptr;
        h.dtype = dtype_from_spec(f[2]);
    } else if (op == "scan" || op == "exclusive_scan" || op == "sort" || op == "unique" ||
               op == "argminmax" || op == "mismatch" || op == "scan_add" ||
               op == "exclusive_scan_shift") {
        if (f.size() != 2) return nullptr;
        h.dtype = dtype_from_spec(f[1]);
        h.kind = op == "scan" ? Kind::SCAN
               : op == "scan_add" ? Kind::SCAN_ADD
               : op == "exclusive_scan" ? Kind::SCAN
               : op == "exclusive_scan_shift" ? Kind::EXSCAN_SHIFT
               : op == "sort" ? Kind::SORT
               : op == "unique" ? Kind::UNIQUE_FLAGS
               : op == "argminmax" ? Kind::ARGMINMAX
               : Kind::MISMATCH;
    } else if (op == "sort_kv") {
        if (f.size() != 2 || f[1] != "u32") return nullptr;
        h.kind = Kind::SORT_KV;
        h.dtype = DType::U64;
    } else if (op == "copy_if" || op == "remove_if" || op == "partition" || op == "count_if" ||
               op == "find") {
        if (f.size() < 3) return nullptr;
        h.dtype = dtype_from_spec(f[1]);
        if (!parse_pred(f, 2, &h.pred)) return nullptr;
        if (h.pred.kind == PredKind::MOD &&
            (h.dtype == DType::F32 || h.dtype == DType::F64))
            return nullptr;
        // a modulus that is zero in a 32-bit element type (x % 0 has no meaning)
        if (h.pred.kind == PredKind::MOD && (h.dtype == DType::I32 || h.dtype == DType::U32) &&
            (uint32_t)h.pred.mod_m == 0)
            return nullptr;
        h.kind = op == "copy_if" ? Kind::COMPACT_FLAGS
               : op == "remove_if" ? Kind::COMPACT_FLAGS
               : op == "partition" ? Kind::PARTITION_SCATTER
               : op == "count_if" ? Kind::COUNT_IF
               : Kind::FIND;
        h.remove = op == "remove_if";
    } else if (op == "map") {
        if (f.size() != 2) return nullptr;
        h.kind = Kind::MAP;
        if (f[1] == "saxpy_gather_f32") { h.map = MapOp::SAXPY_GATHER_F32; h.dtype = DType::F32; }
        else if (f[1] == "affine_f32") { h.map = MapOp::AFFINE_F32; h.dtype = DType::F32; }
        else if (f[1] == "relocate_f32") { h.map = MapOp::DOUBLE_PLUS_ONE_F32; h.dtype = DType::F32; }
        else return nullptr;
    } else {
        return nullptr;
    }
    if (h.dtype == DType::INVALID) return nullptr;
    return intern("spec:" + spec, h);
}

Handle* load_image(const unsigned int* image, size_t words, const std::string& name) {
    if (!image || words == 0) return nullptr;
    if (image[0] == kSpirvMagic) {
        set_error(PARALLAX_ERR_UNSUPPORTED,
                  "kernel '%s' is SPIR-V; this runtime loads sm_100a cubin/fatbin images",
                  name.c_str());
        return nullptr;
    }
    if (image[0] != kElfMagic && image[0] != kFatbinMagic) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "kernel '%s': unknown image format 0x%08x",
                  name.c_str(), image[0]);
        return nullptr;
    }
    if (!ensure_device()) {
        set_error(PARALLAX_ERR_NO_DEVICE, "kernel '%s': no CUDA device", name.c_str());
        return nullptr;
    }
    Handle* h = new Handle();
    h->kind = Kind::USER;
    h->name = name;
    // kept: a transform image may be linked again later, with the fused reduce tile
    const unsigned char* bytes = reinterpret_cast<const unsigned char*>(image);
    h->image.assign(bytes, bytes + words * sizeof(unsigned int));
    if (cudaLibraryLoadData(&h->library, image, nullptr, nullptr, 0, nullptr, nullptr, 0) !=
        cudaSuccess) {
        // relocatable machine code or LTO-IR only: link the image alone, then load that
        cudaGetLastError();
        h->library = nullptr;
        if (!link_images({{h->image.data(), h->image.size()}}, &h->linked, name.c_str()) ||
            !cuda_ok(cudaLibraryLoadData(&h->library, h->linked.data(), nullptr, nullptr, 0,
                                         nullptr, nullptr, 0),
                     "cudaLibraryLoadData")) {
            delete h;
            return nullptr;
        }
    }
    if (!cuda_ok(cudaLibraryGetKernel(&h->kernel, h->library, "parallax_entry"),
                 "cudaLibraryGetKernel(parallax_entry)")) {
        delete h;
        return nullptr;
    }
    return h;
}

}  // namespace

Handle* as_handle(parallax_kernel_t k) { return reinterpret_cast<Handle*>(k); }

Handle* builtin_handle(const char* spec) {
    if (!spec) return nullptr;
    std::lock_guard<std::mutex> g(reg_mu());
    return parse_spec(spec);
}

}  // namespace pxb

using namespace pxb;

PXB_EXPORT parallax_kernel_t parallax_builtin_kernel(const char* spec) {
    Handle* h = builtin_handle(spec);
    if (!h) set_error(PARALLAX_ERR_INVALID_ARGUMENT, "malformed built-in kernel spec '%s'",
                      spec ? spec : "(null)");
    return reinterpret_cast<parallax_kernel_t>(h);
}

PXB_EXPORT parallax_kernel_t parallax_kernel_load(const unsigned int* spirv, size_t words) {
    static std::atomic<uint64_t> counter{0};
    std::string name = "kernel_" + std::to_string(counter.fetch_add(1));
    return reinterpret_cast<parallax_kernel_t>(load_image(spirv, words, name));
}

PXB_EXPORT void parallax_kernel_register(const char* key, const unsigned int* spirv,
                                         size_t words) {
    if (!key) return;
    std::lock_guard<std::mutex> g(reg_mu());
    Entry e;
    e.image = spirv;
    e.words = words;
    registry()[key] = e;
    if (debug()) fprintf(stderr, "[parallax_kernel_register] %s (%zu words)\n", key, words);
}

PXB_EXPORT int parallax_kernel_resolves(const char* key) {
    if (!key) return 0;
    std::lock_guard<std::mutex> g(reg_mu());
    return funnel_builtin(key) != nullptr ? 1 : 0;
}

PXB_EXPORT parallax_kernel_t parallax_kernel_lookup(const char* key) {
    if (!key) return nullptr;
    // Without a device nothing can be launched: every lookup misses and the caller runs its
    // host loop, as a reference lookup does when its kernel cannot be loaded
    // (src/kernel/cache.cpp:90-104).
    if (!ensure_device()) return nullptr;
    std::lock_guard<std::mutex> g(reg_mu());
    auto& reg = registry();
    auto it = reg.find(key);
    if (it != reg.end()) {
        Entry& e = it->second;
        if (!e.resolved) {
            e.resolved = true;
            bool spirv = e.image && e.words && e.image[0] == kSpirvMagic;
            if (!spirv) e.handle = load_image(e.image, e.words, key);
            if (!e.handle) e.handle = funnel_builtin(key);
        }
        if (!e.handle && debug()) fprintf(stderr, "[parallax_kernel_lookup] MISS: %s\n", key);
        return reinterpret_cast<parallax_kernel_t>(e.handle);
    }
    Handle* h = funnel_builtin(key);
    if (!h && debug()) fprintf(stderr, "[parallax_kernel_lookup] MISS: %s\n", key);
    return reinterpret_cast<parallax_kernel_t>(h);
}
