// jit.h -- NVRTC compilation to sm_100a cubins, a disk + memory cache, and
// module/function handles through driver entry points obtained from the
// CUDA runtime (so libnsat.so loads on machines without a driver).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace nsat {

struct DriverApi {
    CUresult (*ModuleLoadData)(CUmodule*, const void*) = nullptr;
    CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*ModuleUnload)(CUmodule) = nullptr;
    CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                             unsigned, CUstream, void**, void**) = nullptr;
    CUresult (*FuncGetAttribute)(int*, CUfunction_attribute, CUfunction) = nullptr;
    CUresult (*GetErrorString)(CUresult, const char**) = nullptr;
    bool ok = false;
};
// Resolves the driver entry points once (after the runtime is initialised).
const DriverApi* driver_api(std::string* err);

struct JitModule {
    CUmodule mod = nullptr;
    std::map<std::string, CUfunction> fns;
    int regs = 0;            // registers per thread of the first kernel
    int local_bytes = 0;     // local (spill) memory per thread
    double compile_ms = 0;   // 0 when loaded from the disk cache
    bool from_disk = false;
    std::string log;
    ~JitModule();
};

// Compiles `src` (or fetches the cubin from the caches) and loads it in the
// current context, which must be `device`'s.  `kernels` are the extern "C"
// names to resolve.  A module stays loaded while the in-memory cache or a
// holder of *out keeps it; release holders with their device current.
int jit_get(int device, const std::string& src, const std::vector<std::string>& kernels, bool verbose,
            std::shared_ptr<JitModule>* out, std::string* err);

// NVRTC compile without loading (no device needed): returns the compile log
// (ptxas resource usage) and the compile time.
int jit_compile_only(const std::string& src, std::string* log, double* ms, std::string* err);

// Directory of the on-disk kernel cache (NSAT_JIT_CACHE, else the user's
// cache directory).
std::string jit_cache_dir();
// The same directory, created if it does not exist yet.
std::string jit_cache_dir_created();

// FNV-1a 64 of a byte string (cache keys).
uint64_t jit_fnv(const std::string& s);


}  // namespace nsat
