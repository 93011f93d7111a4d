// jit.cpp -- NVRTC -> cubin (sm_100a), cached in memory and on disk.
#include "jit.h"
#include "lru.h"

#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace nsat {

namespace {

std::mutex g_mu;
// Loaded modules per device, by source key.  The count is bounded
// (NSAT_JIT_MODULES, default 256): a long-running server compiles a kernel
// for every large QSAT job it tiers, and each stays loaded on the GPU while
// it is cached.  Dropping an entry unloads the module once no circuit handle
// or running solve still holds it.
std::map<int, LruMap<uint64_t, std::shared_ptr<JitModule>>> g_cache;

size_t cache_capacity() {
    static const size_t cap = [] {
        const char* v = getenv("NSAT_JIT_MODULES");
        const long n = v ? atol(v) : 0;
        return n > 0 ? (size_t)n : (size_t)256;
    }();
    return cap;
}

LruMap<uint64_t, std::shared_ptr<JitModule>>& device_cache(int device) {
    auto it = g_cache.find(device);
    if (it == g_cache.end())
        it = g_cache.emplace(device, LruMap<uint64_t, std::shared_ptr<JitModule>>(cache_capacity())).first;
    return it->second;
}
DriverApi g_api;
bool g_api_tried = false;

uint64_t fnv(const std::string& s, uint64_t h = 1469598103934665603ull) {
    for (unsigned char ch : s) { h ^= ch; h *= 1099511628211ull; }
    return h;
}

template <typename F>
bool resolve(const char* name, F* fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
        return false;
    *fn = reinterpret_cast<F>(p);
    return true;
}

std::string cache_dir() {
    const char* e = getenv("NSAT_JIT_CACHE");
    std::string d;
    if (e && *e) d = e;
    else {
        const char* x = getenv("XDG_CACHE_HOME");
        const char* h = getenv("HOME");
        if (x && *x) d = std::string(x) + "/nsat_b200";
        else if (h && *h) d = std::string(h) + "/.cache/nsat_b200";
        else d = "/tmp/nsat_b200";
    }
    return d;
}

void mkdirs(const std::string& d) {
    std::string cur;
    std::stringstream ss(d);
    std::string part;
    if (!d.empty() && d[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

bool read_file(const std::string& p, std::string* out) {
    std::ifstream f(p, std::ios::binary);
    if (!f) return false;
    std::ostringstream s;
    s << f.rdbuf();
    *out = s.str();
    return !out->empty();
}

void write_file_atomic(const std::string& p, const std::string& data) {
    std::string tmp = p + ".tmp." + std::to_string(getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f.write(data.data(), (std::streamsize)data.size());
        if (!f) { unlink(tmp.c_str()); return; }
    }
    if (rename(tmp.c_str(), p.c_str()) != 0) unlink(tmp.c_str());
}

std::string cu_err(CUresult r) {
    const char* s = nullptr;
    if (g_api.GetErrorString) g_api.GetErrorString(r, &s);
    return s ? s : ("CUresult " + std::to_string((int)r));
}

}  // namespace

JitModule::~JitModule() {
    if (mod && g_api.ModuleUnload) g_api.ModuleUnload(mod);
}

const DriverApi* driver_api(std::string* err) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_api_tried) {
        g_api_tried = true;
        bool ok = resolve("cuModuleLoadData", &g_api.ModuleLoadData) &&
                  resolve("cuModuleGetFunction", &g_api.ModuleGetFunction) &&
                  resolve("cuModuleUnload", &g_api.ModuleUnload) &&
                  resolve("cuLaunchKernel", &g_api.LaunchKernel) &&
                  resolve("cuFuncGetAttribute", &g_api.FuncGetAttribute) &&
                  resolve("cuGetErrorString", &g_api.GetErrorString);
        g_api.ok = ok;
    }
    if (!g_api.ok) {
        if (err) *err = "could not resolve CUDA driver entry points";
        return nullptr;
    }
    return &g_api;
}

namespace {
const char* const kOpts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo",
                             "--ptxas-options=-v", "-DNSAT_JIT=1"};
const int kNopts = (int)(sizeof(kOpts) / sizeof(kOpts[0]));

int nvrtc_compile(const std::string& src, std::string* cubin, std::string* log, std::string* err) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "nsat_kernel.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        *err = "nvrtcCreateProgram failed";
        return -3;
    }
    nvrtcResult r = nvrtcCompileProgram(prog, kNopts, kOpts);
    size_t lsz = 0;
    nvrtcGetProgramLogSize(prog, &lsz);
    log->assign(lsz, '\0');
    if (lsz) nvrtcGetProgramLog(prog, &(*log)[0]);
    if (r != NVRTC_SUCCESS) {
        *err = std::string("NVRTC: ") + nvrtcGetErrorString(r) + "\n" + log->substr(0, 4000);
        nvrtcDestroyProgram(&prog);
        return -3;
    }
    size_t csz = 0;
    nvrtcGetCUBINSize(prog, &csz);
    cubin->resize(csz);
    nvrtcGetCUBIN(prog, &(*cubin)[0]);
    nvrtcDestroyProgram(&prog);
    return 0;
}
}  // namespace

int jit_compile_only(const std::string& src, std::string* log, double* ms, std::string* err) {
    auto t0 = std::chrono::steady_clock::now();
    std::string cubin;
    int rc = nvrtc_compile(src, &cubin, log, err);
    *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int jit_get(int device, const std::string& src, const std::vector<std::string>& kernels, bool verbose,
            std::shared_ptr<JitModule>* out, std::string* err) {
    const DriverApi* api = driver_api(err);
    if (!api) return -4;
    int nvmaj = 0, nvmin = 0;
    nvrtcVersion(&nvmaj, &nvmin);
    std::string optstr;
    for (int i = 0; i < kNopts; i++) optstr += std::string(kOpts[i]) + " ";
    const uint64_t key = fnv(src, fnv(optstr + std::to_string(nvmaj) + "." + std::to_string(nvmin)));
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (std::shared_ptr<JitModule>* hit = device_cache(device).find(key)) {
            *out = *hit;
            return 0;
        }
    }
    auto m = std::make_shared<JitModule>();
    char name[64];
    snprintf(name, sizeof(name), "%016llx", (unsigned long long)key);
    if (const char* dump = getenv("NSAT_DUMP_DIR")) {   // generated CUDA source, for inspection
        mkdirs(dump);
        write_file_atomic(std::string(dump) + "/" + name + ".cu", src);
    }
    const std::string dir = cache_dir();
    const std::string cubin_path = dir + "/" + name + ".cubin";
    std::string cubin;
    if (read_file(cubin_path, &cubin)) {
        m->from_disk = true;
        read_file(dir + "/" + name + ".log", &m->log);
    } else {
        auto t0 = std::chrono::steady_clock::now();
        if (int rc = nvrtc_compile(src, &cubin, &m->log, err)) return rc;
        m->compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        mkdirs(dir);
        write_file_atomic(cubin_path, cubin);
        write_file_atomic(dir + "/" + name + ".log", m->log);
    }
    CUresult cr = api->ModuleLoadData(&m->mod, cubin.data());
    if (cr != CUDA_SUCCESS) {
        *err = "cuModuleLoadData: " + cu_err(cr);
        m->mod = nullptr;
        return -3;
    }
    for (const std::string& k : kernels) {
        CUfunction f;
        cr = api->ModuleGetFunction(&f, m->mod, k.c_str());
        if (cr != CUDA_SUCCESS) { *err = "cuModuleGetFunction(" + k + "): " + cu_err(cr); return -3; }
        m->fns[k] = f;
    }
    if (!kernels.empty()) {
        CUfunction f = m->fns[kernels[0]];
        api->FuncGetAttribute(&m->regs, CU_FUNC_ATTRIBUTE_NUM_REGS, f);
        api->FuncGetAttribute(&m->local_bytes, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, f);
    }
    if (verbose)
        fprintf(stderr, "[nsat] jit %s: %s regs=%d local=%dB compile=%.1fms\n", name,
                m->from_disk ? "disk" : "nvrtc", m->regs, m->local_bytes, m->compile_ms);
    // modules evicted to make room are released when this function returns:
    // outside the lock, with this device current (the caller's contract)
    std::vector<std::shared_ptr<JitModule>> evicted;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        device_cache(device).put(key, m, &evicted);
    }
    *out = m;
    return 0;
}

std::string jit_cache_dir() { return cache_dir(); }

std::string jit_cache_dir_created() {
    const std::string d = cache_dir();
    mkdirs(d);
    return d;
}

uint64_t jit_fnv(const std::string& s) { return fnv(s); }

}  // namespace nsat
