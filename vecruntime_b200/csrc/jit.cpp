// Per-spec aggregate kernels: the kernel source (agg_main.cuh and the headers
// it includes, embedded at build time) compiled with NVRTC for sm_100a, with
// the spec's Program written out as a compile-time constant (kJitProg). All
// op and key loops then unroll and every op's kind, columns and word offsets
// become immediates: a few tens of instructions per row instead of an
// interpreter's hundreds. NVRTC is opened with dlopen and the driver module
// API reached through cudaGetDriverEntryPoint, so the library has no
// link-time dependency on either; without them the ahead-of-time
// (interpreted) kernel runs instead.
#include "jit.h"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

#include "jit_sources.inc"

namespace vr {

struct JitKernel {
    CUmodule mod = nullptr;
    CUfunction fn = nullptr;
    int regs = 0;
    int smem_set = 0;
    int threads = 0;  // consumer threads it was compiled for (a compile-time constant inside)
};

namespace {

struct Nvrtc {
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    bool ok = false;
    std::string why;
};

Nvrtc& nvrtc() {
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* name : names)
            if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            const char* e = dlerror();
            n.why = std::string("NVRTC not found: ") + (e ? e : "");
            return;
        }
        n.create = (decltype(n.create))dlsym(h, "nvrtcCreateProgram");
        n.compile = (decltype(n.compile))dlsym(h, "nvrtcCompileProgram");
        n.log_size = (decltype(n.log_size))dlsym(h, "nvrtcGetProgramLogSize");
        n.log = (decltype(n.log))dlsym(h, "nvrtcGetProgramLog");
        n.cubin_size = (decltype(n.cubin_size))dlsym(h, "nvrtcGetCUBINSize");
        n.cubin = (decltype(n.cubin))dlsym(h, "nvrtcGetCUBIN");
        n.destroy = (decltype(n.destroy))dlsym(h, "nvrtcDestroyProgram");
        n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
        if (!n.ok) n.why = "NVRTC entry points missing";
    });
    return n;
}

typedef CUresult (*PFN_load)(CUmodule*, const void*);
typedef CUresult (*PFN_getfn)(CUfunction*, CUmodule, const char*);
typedef CUresult (*PFN_setattr)(CUfunction, CUfunction_attribute, int);
typedef CUresult (*PFN_getattr)(int*, CUfunction_attribute, CUfunction);
typedef CUresult (*PFN_launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               CUstream, void**, void**);

struct Driver {
    PFN_load load = nullptr;
    PFN_getfn getfn = nullptr;
    PFN_setattr setattr = nullptr;
    PFN_getattr getattr = nullptr;
    PFN_launch launch = nullptr;
    bool ok = false;
};

Driver& driver() {
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        auto get = [](const char* sym) -> void* {
            void* p = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint(sym, &p, cudaEnableDefault, &q) != cudaSuccess ||
                q != cudaDriverEntryPointSuccess)
                return nullptr;
            return p;
        };
        d.load = (PFN_load)get("cuModuleLoadData");
        d.getfn = (PFN_getfn)get("cuModuleGetFunction");
        d.setattr = (PFN_setattr)get("cuFuncSetAttribute");
        d.getattr = (PFN_getattr)get("cuFuncGetAttribute");
        d.launch = (PFN_launch)get("cuLaunchKernel");
        d.ok = d.load && d.getfn && d.setattr && d.getattr && d.launch;
    });
    return d;
}

const char* kPrelude =
    "typedef signed char int8_t;\n"
    "typedef unsigned char uint8_t;\n"
    "typedef short int16_t;\n"
    "typedef unsigned short uint16_t;\n"
    "typedef int int32_t;\n"
    "typedef unsigned int uint32_t;\n"
    "typedef long long int64_t;\n"
    "typedef unsigned long long uint64_t;\n"
    "typedef unsigned long uintptr_t;\n"
    "#define VR_JIT 1\n";

// The Program as a C++ aggregate initializer (field order of vr_internal.h).
std::string program_literal(const Program& P) {
    std::ostringstream o;
    auto arr_u8 = [&](const uint8_t* a, int n) {
        o << "{";
        for (int i = 0; i < n; ++i) o << (int)a[i] << (i + 1 < n ? "," : "");
        o << "}";
    };
    o << "{" << P.num_cols << ",";
    arr_u8(P.col_lane, kMaxCols);
    o << ",";
    arr_u8(P.col_width, kMaxCols);
    o << ",";
    arr_u8(P.col_nullable, kMaxCols);
    o << "," << P.num_keys << ",{";
    for (int k = 0; k < kMaxKeys; ++k) {
        const KeyField& f = P.keys[k];
        o << "{" << (int)f.col << "," << (int)f.lane << "," << (int)f.word << "," << (int)f.shift << "," << (int)f.bits
          << "," << (int)f.null_word << "," << (int)f.null_shift << "," << (int)f.remap << "," << f.card << "," << f.pad2
          << "," << (long long)f.mul << "LL}" << (k + 1 < kMaxKeys ? "," : "");
    }
    o << "}," << P.kw << "," << P.occ_word << "," << P.occ_shift << "," << P.lock_mode << "," << P.aw << "," << P.sw
      << "," << P.hw << "," << P.num_ops << ",{";
    for (int i = 0; i < kMaxOps; ++i) {
        const OpDesc& d = P.ops[i];
        o << "{" << (int)d.kind << "," << (int)d.lane << "," << (int)d.flags << "," << (int)d.nwords << ","
          << (int)d.col << "," << (int)d.col2 << "," << (int)d.nterms << "," << (int)d.prec << "," << d.word << ","
          << d.hword << ",{" << (int)d.term_col[0] << "," << (int)d.term_col[1] << "," << (int)d.term_col[2] << "},{"
          << (int)d.term_sign[0] << "," << (int)d.term_sign[1] << "," << (int)d.term_sign[2] << "}," << d.prefix_op << ",{"
          << (long long)d.term_add[0] << "LL," << (long long)d.term_add[1] << "LL," << (long long)d.term_add[2]
          << "LL}}" << (i + 1 < kMaxOps ? "," : "");
    }
    o << "},";
    arr_u8(P.word_kind, kMaxAccWords);
    o << "," << (long long)P.direct_slots << "LL}";
    return o.str();
}

std::string key_literal(const KeyField& f) {
    std::ostringstream o;
    o << "{" << (int)f.col << "," << (int)f.lane << "," << (int)f.word << "," << (int)f.shift << "," << (int)f.bits << ","
      << (int)f.null_word << "," << (int)f.null_shift << "," << (int)f.remap << "," << f.card << "," << f.pad2 << ","
      << (long long)f.mul << "LL}";
    return o.str();
}

std::string op_literal(const OpDesc& d) {
    std::ostringstream o;
    o << "{" << (int)d.kind << "," << (int)d.lane << "," << (int)d.flags << "," << (int)d.nwords << "," << (int)d.col
      << "," << (int)d.col2 << "," << (int)d.nterms << "," << (int)d.prec << "," << d.word << "," << d.hword << ",{"
      << (int)d.term_col[0] << "," << (int)d.term_col[1] << "," << (int)d.term_col[2] << "},{" << (int)d.term_sign[0]
      << "," << (int)d.term_sign[1] << "," << (int)d.term_sign[2] << "}," << d.prefix_op << ",{" << (long long)d.term_add[0]
      << "LL," << (long long)d.term_add[1] << "LL," << (long long)d.term_add[2] << "LL}}";
    return o.str();
}

// The per-spec hooks agg_main.cuh calls under VR_JIT: each key field and
// each op as its own statement with compile-time constant descriptors.
std::string hooks(const Program& P) {
    std::ostringstream o;
    o << "namespace vr {\n";
    o << "template <bool SM>\nVR_DEV int jit_direct_index(const TileView& v, int64_t r) {\n  int idx = 0;\n";
    for (int f = 0; f < P.num_keys; ++f)
        o << "  { constexpr KeyField kf = " << key_literal(P.keys[f])
          << "; int x = direct_field32<SM>(kf, v, r); if (x < 0) return -1; idx += x; }\n";
    o << "  return idx;\n}\n";
    o << "template <int KW>\nVR_DEV void jit_pack_key(const TileView& v, int64_t r, uint64_t (&k)[KW], bool& side, "
         "bool& bad) {\n#pragma unroll\n  for (int i = 0; i < KW; ++i) k[i] = 0;\n  side = false;\n  bad = false;\n";
    for (int f = 0; f < P.num_keys; ++f)
        o << "  { constexpr KeyField kf = " << key_literal(P.keys[f]) << "; pack_field<KW>(kf, v, r, k, bad); }\n";
    o << "  pack_finish<KW>(" << P.occ_word << ", " << P.occ_shift << ", k, side);\n}\n";
    o << "template <class F>\nVR_DEV void jit_for_op(int i, F&& f) {\n  switch (i) {\n";
    for (int i = 0; i < P.num_ops; ++i)
        o << "    case " << i << ": { constexpr OpDesc op = " << op_literal(P.ops[i]) << "; f(op, KindTag<"
          << (int)P.ops[i].kind << ">{}); break; }\n";
    o << "  }\n}\n}  // namespace vr\n";
    return o.str();
}

uint64_t fnv64(const std::string& s) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 0x100000001b3ull;
    }
    return h;
}

std::mutex g_mu;
std::map<std::pair<int, uint64_t>, JitKernel*> g_cache;  // (device, source hash)

// `verbose`: ptxas resource usage (registers, spills, local memory) is
// returned in *err on success too.
bool compile_cubin(const std::string& src, std::vector<char>& cubin, std::string* err, bool verbose = false) {
    Nvrtc& n = nvrtc();
    if (!n.ok) {
        *err = n.why;
        return false;
    }
    nvrtcProgram prog;
    if (n.create(&prog, src.c_str(), "vr_jit_aggregate.cu", jitsrc::kNum, jitsrc::kTexts, jitsrc::kNames) !=
        NVRTC_SUCCESS) {
        *err = "nvrtcCreateProgram failed";
        return false;
    }
    // -default-device: the ABI's host prototypes in vrgpu.h are declarations
    // only here (never defined or called)
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-DVR_JIT=1", "-default-device",
                          "--device-int128", "--ptxas-options=-v"};
    nvrtcResult r = n.compile(prog, verbose ? 7 : 6, opts);
    if (r != NVRTC_SUCCESS) {
        size_t ls = 0;
        n.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) n.log(prog, &log[0]);
        *err = "NVRTC compile failed: " + log.substr(0, 2000);
        n.destroy(&prog);
        return false;
    }
    if (verbose) {
        size_t ls = 0;
        n.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) n.log(prog, &log[0]);
        *err = log;
    }
    size_t cs = 0;
    n.cubin_size(prog, &cs);
    cubin.resize(cs);
    n.cubin(prog, cubin.data());
    n.destroy(&prog);
    return true;
}

}  // namespace

bool jit_enabled() {
    const char* e = std::getenv("VRGPU_JIT");
    return !(e && std::strcmp(e, "0") == 0);
}

static std::string jit_source(const Program& P, const JitShape& S) {
    std::string src = kPrelude;
    src += "#define VR_JIT_KW " + std::to_string(S.kw) + "\n#define VR_JIT_TIER " + std::to_string(S.tier) + "\n";
    src += "#define VR_JIT_RCHUNK " + std::to_string(S.rchunk) + "\n";
    src += "#define VR_JIT_WARP_AGG " + std::to_string(S.warp_agg ? 1 : 0) + "\n";
    src += "#define VR_JIT_THREADS " + std::to_string(S.threads) + "\n";
    src += "#define VR_JIT_HW " + std::to_string(P.hw) + "\n#define VR_JIT_AW " + std::to_string(P.aw) + "\n";
    src += "#define VR_JIT_SW " + std::to_string(P.sw) + "\n#define VR_JIT_DSLOTS " +
           std::to_string((long long)P.direct_slots) + "LL\n";
    src += "#define VR_JIT_NUM_OPS " + std::to_string(P.num_ops) + "\n";
    src += "#include \"agg_device.cuh\"\nnamespace vr {\n__constant__ const Program kJitProg = ";
    src += program_literal(P);
    src += ";\n}\n#include \"agg_main.cuh\"\n";
    src += hooks(P);
    src +=
        "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(S.threads + 32) + ", " +
        std::to_string(S.min_blocks) + ")\n"
        "vr_jit_aggregate(const vr::BatchDesc* __restrict__ descs, const vr::LaunchCfg cfg,\n"
        "                 unsigned long long* __restrict__ tile_counter) {\n"
        "    extern __shared__ __align__(128) unsigned char smem[];\n"
        "    vr::aggregate_body<VR_JIT_KW, VR_JIT_TIER>(descs, cfg, (uint64_t*)tile_counter, smem);\n"
        "}\n";
    return src;
}

bool jit_compile_only(const Program& P, const JitShape& S, size_t* cubin_bytes, std::string* err) {
    std::vector<char> cubin;
    if (!compile_cubin(jit_source(P, S), cubin, err, true)) return false;
    if (cubin_bytes) *cubin_bytes = cubin.size();
    return true;
}

JitKernel* jit_get(const Program& P, const JitShape& S, int device, std::string* err) {
    std::string src = jit_source(P, S);
    uint64_t h = fnv64(src);
    for (int i = 0; i < jitsrc::kNum; ++i) h ^= fnv64(jitsrc::kTexts[i]) * (i + 3);
    std::lock_guard<std::mutex> lk(g_mu);
    auto key = std::make_pair(device, h);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;
    Driver& d = driver();
    if (!d.ok) {
        *err = "CUDA driver module API unavailable";
        return nullptr;
    }
    std::vector<char> cubin;
    std::string path;
    if (const char* dir = std::getenv("VRGPU_JIT_CACHE")) {
        char name[64];
        std::snprintf(name, sizeof(name), "/vrjit_%016llx.cubin", (unsigned long long)h);
        path = std::string(dir) + name;
        std::ifstream f(path, std::ios::binary);
        if (f) cubin.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    if (cubin.empty()) {
        if (!compile_cubin(src, cubin, err)) return nullptr;
        if (!path.empty()) {
            std::ofstream f(path, std::ios::binary);
            f.write(cubin.data(), (std::streamsize)cubin.size());
        }
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaFree(nullptr);  // the primary context is current for the driver calls below
    JitKernel* k = new JitKernel();
    CUresult r = d.load(&k->mod, cubin.data());
    if (r == CUDA_SUCCESS) r = d.getfn(&k->fn, k->mod, "vr_jit_aggregate");
    if (r == CUDA_SUCCESS) r = d.getattr(&k->regs, CU_FUNC_ATTRIBUTE_NUM_REGS, k->fn);
    k->threads = S.threads;
    cudaSetDevice(prev);
    if (r != CUDA_SUCCESS) {
        *err = "loading the compiled kernel failed (CUresult " + std::to_string((int)r) + ")";
        delete k;
        return nullptr;
    }
    g_cache[key] = k;
    return k;
}

int jit_regs(const JitKernel* k) { return k ? k->regs : 0; }

cudaError_t jit_launch(JitKernel* k, const BatchDesc* descs, const LaunchCfg& cfg, int blocks, uint64_t* tile_counter,
                       cudaStream_t stream) {
    Driver& d = driver();
    if (cfg.consumer_threads != k->threads) return cudaErrorInvalidConfiguration;  // compiled for another shape
    if (k->smem_set < cfg.smem_bytes) {
        if (d.setattr(k->fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, cfg.smem_bytes) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
        k->smem_set = cfg.smem_bytes;
    }
    LaunchCfg c = cfg;
    const BatchDesc* dp = descs;
    uint64_t* tc = tile_counter;
    void* params[] = {(void*)&dp, (void*)&c, (void*)&tc};
    CUresult r = d.launch(k->fn, (unsigned)blocks, 1, 1, (unsigned)(cfg.consumer_threads + 32), 1, 1,
                          (unsigned)cfg.smem_bytes, (CUstream)stream, params, nullptr);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

}  // namespace vr
