// User step hooks: the plugin's __device__ step() compiled at run time.
//
// The reference builds its kernels from the plugin's .cu file when a Solver
// starts (pysweep/core/io.py:146-155: SourceModule(pysweep.cu with
// -DPYSWEEP_GPU_SOURCE=<file>)) and copies the framework and plugin constants
// into the module's __constant__ variables by name (io.py:169-184,
// pysweep/equations/heat.py:38-46).  This file does the same with NVRTC for
// sm_100a: the hook's source is wrapped in the program of hook_program(),
// whose kernels (hook_kernels.cuh) run it inside the swept phases and a tiled
// standard step; the module is loaded with the driver API into the current
// (primary) context; constants are found by name in the three kernel-kind
// namespaces.  NVRTC is opened with dlopen on first use and the driver-API
// calls are resolved through the runtime (cudaGetDriverEntryPoint), so the
// library loads (and every built-in equation runs) where NVRTC is absent, and
// loads without a driver at all on a machine with no GPU.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace psb {

// kernel kinds, each with its own namespace, tile geometry and constants
enum HookNs { HOOK_STREAM = 0, HOOK_SEAM = 1, HOOK_STD = 2 };
constexpr const char* kHookNs[3] = {"psh_stream", "psh_seam", "psh_std"};
// framework constants of pysweep/core/pysweep.cu:12-20, in this order
enum HookFw { FW_VARS, FW_TIMES, FW_MPSS, FW_MOSS, FW_NV, FW_OPS, FW_ITS, FW_SX, FW_SY, FW_COUNT };
constexpr const char* kHookFw[FW_COUNT] = {"VARS", "TIMES", "MPSS", "MOSS", "NV",
                                           "OPS",  "ITS",   "SX",   "SY"};
// standard-step tile of the hook kernels (hook_kernels.cuh)
constexpr int kHookStdTR = 16, kHookStdTC = 32, kHookStdNT = 256;

// A user constant, in every namespace (ps_get_global hands out a pointer to
// it; `name` comes first, as in the built-in constants' table).
struct HookConst {
    const char* name = nullptr;
    size_t size = 0;
    CUdeviceptr ptr[3] = {0, 0, 0};
};

struct HookModule {
    CUmodule mod = nullptr;
    CUfunction prism[2] = {nullptr, nullptr};  // chunk 32, 64
    CUfunction gap[2] = {nullptr, nullptr};
    CUfunction ybridge = nullptr, octahedron = nullptr, standard = nullptr;
    CUdeviceptr fw[3][FW_COUNT] = {};
    int fw_val[3][FW_COUNT];  // last values written (-1: never)
    std::map<std::string, HookConst> consts;
    int nv = 1, ops = 1, its = 1;
    size_t std_smem = 0;
    HookModule()
    {
        for (auto& r : fw_val)
            for (int& v : r) v = -1;
    }
};

// ------------------------------------------------------------- driver API --
// The driver calls the hook path makes, resolved once from the driver the
// CUDA runtime loaded.
struct Driver {
    decltype(&cuModuleLoadData) moduleLoadData = nullptr;
    decltype(&cuModuleUnload) moduleUnload = nullptr;
    decltype(&cuModuleGetFunction) moduleGetFunction = nullptr;
    decltype(&cuModuleGetGlobal) moduleGetGlobal = nullptr;
    decltype(&cuFuncSetAttribute) funcSetAttribute = nullptr;
    decltype(&cuMemcpyHtoDAsync) memcpyHtoDAsync = nullptr;
    decltype(&cuLaunchKernel) launchKernel = nullptr;
    decltype(&cuGetErrorString) getErrorString = nullptr;
    bool ok = false;
};

inline Driver& drv()
{
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        auto get = [](const char* sym, void** fn) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPoint(sym, fn, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *fn;
        };
        d.ok = get("cuModuleLoadData", (void**)&d.moduleLoadData) &&
               get("cuModuleUnload", (void**)&d.moduleUnload) &&
               get("cuModuleGetFunction", (void**)&d.moduleGetFunction) &&
               get("cuModuleGetGlobal", (void**)&d.moduleGetGlobal) &&
               get("cuFuncSetAttribute", (void**)&d.funcSetAttribute) &&
               get("cuMemcpyHtoDAsync", (void**)&d.memcpyHtoDAsync) &&
               get("cuLaunchKernel", (void**)&d.launchKernel) &&
               get("cuGetErrorString", (void**)&d.getErrorString);
    });
    return d;
}

// ------------------------------------------------------------------ NVRTC --
// The handful of NVRTC entry points used, resolved from the shared library.
struct Nvrtc {
    using Create = int (*)(void**, const char*, const char*, int, const char* const*,
                           const char* const*);
    using Compile = int (*)(void*, int, const char* const*);
    using Size = int (*)(void*, size_t*);
    using Get = int (*)(void*, char*);
    using Destroy = int (*)(void**);
    Create create = nullptr;
    Compile compile = nullptr;
    Size log_size = nullptr, cubin_size = nullptr;
    Get log = nullptr, cubin = nullptr;
    Destroy destroy = nullptr;
    bool ok = false;
    std::string why;
};

inline Nvrtc& nvrtc()
{
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* home = getenv("CUDA_HOME");
        std::vector<std::string> names = {"libnvrtc.so.12", "libnvrtc.so"};
        names.push_back(std::string(home ? home : "/usr/local/cuda") + "/lib64/libnvrtc.so.12");
        void* h = nullptr;
        for (const auto& nm : names)
            if ((h = dlopen(nm.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            n.why = "libnvrtc.so.12 not found (needed to compile step hooks)";
            return;
        }
        n.create = (Nvrtc::Create)dlsym(h, "nvrtcCreateProgram");
        n.compile = (Nvrtc::Compile)dlsym(h, "nvrtcCompileProgram");
        n.log_size = (Nvrtc::Size)dlsym(h, "nvrtcGetProgramLogSize");
        n.log = (Nvrtc::Get)dlsym(h, "nvrtcGetProgramLog");
        n.cubin_size = (Nvrtc::Size)dlsym(h, "nvrtcGetCUBINSize");
        n.cubin = (Nvrtc::Get)dlsym(h, "nvrtcGetCUBIN");
        n.destroy = (Nvrtc::Destroy)dlsym(h, "nvrtcDestroyProgram");
        n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
        if (!n.ok) n.why = "libnvrtc lacks an entry point";
    });
    return n;
}

// Directory of this library's kernel headers (csrc/ beside the .so).
inline std::string hook_include_dir()
{
    Dl_info info;
    if (dladdr((void*)&hook_include_dir, &info) && info.dli_fname) {
        std::string p = info.dli_fname;
        const size_t k = p.rfind('/');
        return (k == std::string::npos ? std::string(".") : p.substr(0, k)) + "/csrc";
    }
    return "csrc";
}

// The run-time program: the hook once per kernel kind, each copy in a
// namespace that declares the framework constants as the reference's
// pysweep.cu does (so the hook's VARS, TIMES, SY, ... resolve to them), then
// the kernels.
inline std::string hook_program(const std::string& src, const std::string& name, int nv, int ops,
                                int its)
{
    std::string p;
    p += "#define PSH_NV " + std::to_string(nv) + "\n";
    p += "#define PSH_OPS " + std::to_string(ops) + "\n";
    p += "#define PSH_ITS " + std::to_string(its) + "\n";
    p += "#define PSH_STD_TR " + std::to_string(kHookStdTR) + "\n";
    p += "#define PSH_STD_TC " + std::to_string(kHookStdTC) + "\n";
    p += "#define PSH_STD_NT " + std::to_string(kHookStdNT) + "\n";
    for (const char* ns : kHookNs) {
        p += std::string("namespace ") + ns + " {\n";
        p += "__device__ __constant__ int VARS, TIMES, MPSS, MOSS, NV, OPS, ITS, SX, SY;\n";
        p += "__device__ __constant__ const int LB_MIN_BLOCKS = 1;\n";
        p += "__device__ __constant__ const int LB_MAX_THREADS = 1024;\n";
        p += "#line 1 \"" + name + "\"\n";
        p += src;
        p += "\n}\n";
    }
    p += "#include \"hook_kernels.cuh\"\n";
    return p;
}

// Compile a program for sm_100a into a cubin; returns 0 or PS_ERR_* with the
// compiler's log in *log.  Cubins are cached per program text.
inline int hook_compile(const std::string& prog, std::vector<char>* cubin, std::string* log)
{
    static std::mutex mu;
    static std::map<std::string, std::vector<char>> cache;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(prog);
        if (it != cache.end()) {
            *cubin = it->second;
            return 0;
        }
    }
    Nvrtc& n = nvrtc();
    if (!n.ok) {
        *log = n.why;
        return -6;  // PS_ERR_COMPILE
    }
    void* h = nullptr;
    if (n.create(&h, prog.c_str(), "pysweep_hook.cu", 0, nullptr, nullptr) != 0) {
        *log = "nvrtcCreateProgram failed";
        return -6;
    }
    const std::string inc = "-I" + hook_include_dir();
    const char* opts[] = {"-arch=sm_100a", "--fmad=false", "-std=c++17", "-lineinfo",
                          "-diag-suppress=177,550", inc.c_str()};
    const int rc = n.compile(h, (int)(sizeof opts / sizeof *opts), opts);
    size_t ls = 0;
    n.log_size(h, &ls);
    std::string lg(ls, '\0');
    if (ls) n.log(h, &lg[0]);
    while (!lg.empty() && (lg.back() == '\0' || lg.back() == '\n')) lg.pop_back();
    *log = lg;
    if (rc != 0) {
        n.destroy(&h);
        return -6;
    }
    size_t cs = 0;
    n.cubin_size(h, &cs);
    cubin->assign(cs, 0);
    n.cubin(h, cubin->data());
    n.destroy(&h);
    std::lock_guard<std::mutex> lock(mu);
    cache[prog] = *cubin;
    return 0;
}

// Itanium name of the namespace-scope variable ns::name (what the module's
// symbol table holds for a __constant__ declared inside a namespace).
inline std::string hook_mangle(const char* ns, const std::string& name)
{
    return "_ZN" + std::to_string(strlen(ns)) + ns + std::to_string(name.size()) + name + "E";
}

inline std::string cu_error(CUresult r)
{
    const char* s = nullptr;
    if (drv().getErrorString) drv().getErrorString(r, &s);
    return s ? s : "CUDA driver error " + std::to_string((int)r);
}

// Load a compiled hook module into the current context and resolve its
// kernels and framework constants.
inline int hook_load(HookModule* h, const std::vector<char>& cubin, std::string* err)
{
    Driver& d = drv();
    if (!d.ok) {
        *err = "the CUDA driver API entry points are unavailable";
        return -2;
    }
    CUresult r = d.moduleLoadData(&h->mod, cubin.data());
    if (r != CUDA_SUCCESS) {
        *err = "cuModuleLoadData: " + cu_error(r);
        return -2;
    }
    const char* names[] = {"psh_prism32", "psh_prism64", "psh_gap32", "psh_gap64",
                           "psh_ybridge", "psh_octahedron", "psh_standard"};
    CUfunction* dst[] = {&h->prism[0], &h->prism[1], &h->gap[0], &h->gap[1],
                         &h->ybridge,  &h->octahedron, &h->standard};
    for (int i = 0; i < 7; ++i) {
        r = d.moduleGetFunction(dst[i], h->mod, names[i]);
        if (r == CUDA_SUCCESS)
            r = d.funcSetAttribute(*dst[i], CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                   227 * 1024);
        if (r != CUDA_SUCCESS) {
            *err = std::string(names[i]) + ": " + cu_error(r);
            return -2;
        }
    }
    for (int k = 0; k < 3; ++k)
        for (int f = 0; f < FW_COUNT; ++f) {
            size_t sz = 0;
            r = d.moduleGetGlobal(&h->fw[k][f], &sz, h->mod,
                                  hook_mangle(kHookNs[k], kHookFw[f]).c_str());
            if (r != CUDA_SUCCESS) {
                *err = std::string("framework constant ") + kHookFw[f] + ": " + cu_error(r);
                return -2;
            }
        }
    return 0;
}

// Find a user constant by name in the module (every namespace holds a copy);
// nullptr when the hook declares no such __constant__.
inline HookConst* hook_const(HookModule* h, const std::string& name)
{
    auto it = h->consts.find(name);
    if (it != h->consts.end()) return &it->second;
    for (int f = 0; f < FW_COUNT; ++f)
        if (name == kHookFw[f]) return nullptr;  // framework constants are not the plugin's
    HookConst c;
    for (int k = 0; k < 3; ++k) {
        size_t sz = 0;
        if (drv().moduleGetGlobal(&c.ptr[k], &sz, h->mod, hook_mangle(kHookNs[k], name).c_str()) !=
            CUDA_SUCCESS)
            return nullptr;
        c.size = sz;
    }
    auto ins = h->consts.emplace(name, c).first;
    ins->second.name = ins->first.c_str();
    return &ins->second;
}

// Write a framework constant of one namespace in stream order (skipped when
// it already holds the value).
inline CUresult hook_set_fw(HookModule* h, int ns, int f, int value, CUstream st)
{
    if (h->fw_val[ns][f] == value) return CUDA_SUCCESS;
    CUresult r = drv().memcpyHtoDAsync(h->fw[ns][f], &value, sizeof(int), st);
    if (r == CUDA_SUCCESS) h->fw_val[ns][f] = value;
    return r;
}

}  // namespace psb
