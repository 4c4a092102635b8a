// Run-time compilation of kernels specialised to one stencil.
//
// The reference turns every stencil function into its own CUDA kernel at
// translation time (translator/cuda_translator.cc:615-869). A registered
// psb_generic_stencil arrives as a term table at run time instead, so the
// library compiles its kernel then: the source is the library's own device
// headers (k_generic_tma.cuh and what it includes, read from the csrc/
// directory beside the library) plus a generated term program, compiled by
// NVRTC for sm_100a and loaded as a module of the current context. NVRTC is
// opened with dlopen, so the library loads and runs without it (the caller
// then keeps the kernel that interprets the table). Functions are cached per
// (device, key) for the life of the process.
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace psb {

namespace {

struct NvrtcApi {
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

typedef CUresult (*ModuleLoadDataFn)(CUmodule *, const void *);
typedef CUresult (*ModuleGetFunctionFn)(CUfunction *, CUmodule, const char *);
typedef CUresult (*FuncSetAttributeFn)(CUfunction, CUfunction_attribute, int);
typedef CUresult (*LaunchKernelFn)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned,
                                   unsigned, unsigned, CUstream, void **, void **);

struct DriverApi {
  ModuleLoadDataFn load = nullptr;
  ModuleGetFunctionFn get = nullptr;
  FuncSetAttributeFn set_attr = nullptr;
  LaunchKernelFn launch = nullptr;
};

template <typename F>
bool sym(void *h, const char *name, F *out) {
  *out = reinterpret_cast<F>(dlsym(h, name));
  return *out != nullptr;
}

const NvrtcApi *nvrtc_api() {
  static NvrtcApi api;
  static bool tried = false, ok = false;
  if (tried) return ok ? &api : nullptr;
  tried = true;
  const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12",
                         "/usr/local/cuda/lib64/libnvrtc.so"};
  void *h = nullptr;
  for (const char *n : names)
    if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
  if (!h) return nullptr;
  ok = sym(h, "nvrtcCreateProgram", &api.create) && sym(h, "nvrtcCompileProgram", &api.compile) &&
       sym(h, "nvrtcGetProgramLogSize", &api.log_size) &&
       sym(h, "nvrtcGetProgramLog", &api.log) && sym(h, "nvrtcGetCUBINSize", &api.cubin_size) &&
       sym(h, "nvrtcGetCUBIN", &api.cubin) && sym(h, "nvrtcDestroyProgram", &api.destroy);
  return ok ? &api : nullptr;
}

template <typename F>
bool driver_sym(const char *name, F *out) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return false;
  *out = reinterpret_cast<F>(p);
  return true;
}

const DriverApi *driver_api() {
  static DriverApi api;
  static bool tried = false, ok = false;
  if (tried) return ok ? &api : nullptr;
  tried = true;
  ok = driver_sym("cuModuleLoadData", &api.load) &&
       driver_sym("cuModuleGetFunction", &api.get) &&
       driver_sym("cuFuncSetAttribute", &api.set_attr) &&
       driver_sym("cuLaunchKernel", &api.launch);
  return ok ? &api : nullptr;
}

// The library's device headers: $PHYSIS_B200_CSRC, else csrc/ beside the
// directory that holds this library (physis_b200/lib -> physis_b200/csrc).
std::string csrc_dir() {
  if (const char *e = getenv("PHYSIS_B200_CSRC")) return e;
  Dl_info info;
  if (!dladdr(reinterpret_cast<void *>(&csrc_dir), &info) || !info.dli_fname) return "";
  std::string p = info.dli_fname;
  const size_t slash = p.rfind('/');
  if (slash == std::string::npos) return "";
  p = p.substr(0, slash);  // .../lib
  const size_t up = p.rfind('/');
  if (up == std::string::npos) return "";
  return p.substr(0, up) + "/csrc";
}

// Types and macros the device headers take from host headers, for the
// run-time compiler (which has no system headers).
std::string prelude() {
  std::string s =
      "typedef signed char int8_t;\ntypedef unsigned char uint8_t;\n"
      "typedef short int16_t;\ntypedef unsigned short uint16_t;\n"
      "typedef int int32_t;\ntypedef unsigned int uint32_t;\n"
      "typedef long long int64_t;\ntypedef unsigned long long uint64_t;\n"
      "typedef unsigned long size_t;\ntypedef unsigned long uintptr_t;\n"
      "struct __align__(64) CUtensorMap_st { unsigned long long opaque[16]; };\n"
      "typedef CUtensorMap_st CUtensorMap;\n";
  s += "#define PSB_MAX_TERMS " + std::to_string(PSB_MAX_TERMS) + "\n";
  s += "#define PSB_MAX_GRIDS " + std::to_string(PSB_MAX_GRIDS) + "\n";
  return s;
}

static_assert(sizeof(CUtensorMap) == 128 && alignof(CUtensorMap) == 64,
              "the prelude's tensor-map type must match cuda.h");

std::mutex g_mu;
std::map<std::string, CUfunction> g_cache;  // device + key -> function (nullptr: failed)

}  // namespace

bool rtc_available() { return nvrtc_api() && driver_api() && !csrc_dir().empty(); }

psb_status rtc_function(const std::string &key, const std::string &source, const char *name,
                        const std::vector<std::string> &options, int smem_bytes,
                        CUfunction *fn) {
  *fn = nullptr;
  const NvrtcApi *nv = nvrtc_api();
  const DriverApi *dr = driver_api();
  if (!nv || !dr) return PSB_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PSB_ERR_CUDA;
  const std::string ckey = std::to_string(dev) + "|" + key;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(ckey);
  if (it != g_cache.end()) {
    *fn = it->second;
    return *fn ? PSB_OK : PSB_ERR_UNSUPPORTED;
  }
  g_cache[ckey] = nullptr;  // a failed compile is not retried
  const std::string dir = csrc_dir();
  if (dir.empty()) return PSB_ERR_UNSUPPORTED;
  std::vector<std::string> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false",
                                   "-default-device", "-I" + dir};
  opts.insert(opts.end(), options.begin(), options.end());
  std::vector<const char *> optp;
  for (const auto &o : opts) optp.push_back(o.c_str());
  const std::string pre = prelude();
  const char *hdr_src[] = {pre.c_str()};
  const char *hdr_name[] = {"psb_rtc_prelude.h"};
  nvrtcProgram prog = nullptr;
  if (nv->create(&prog, source.c_str(), "psb_stencil.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS)
    return PSB_ERR_UNSUPPORTED;
  const nvrtcResult cr = nv->compile(prog, (int)optp.size(), optp.data());
  if (cr != NVRTC_SUCCESS) {
    size_t n = 0;
    nv->log_size(prog, &n);
    std::string log(n, '\0');
    if (n) nv->log(prog, &log[0]);
    if (__ps_trace)
      fprintf(__ps_trace, "physis_b200: run-time compilation of %s failed:\n%s\n", name,
              log.c_str());
    nv->destroy(&prog);
    return PSB_ERR_UNSUPPORTED;
  }
  size_t nbin = 0;
  nv->cubin_size(prog, &nbin);
  std::vector<char> bin(nbin);
  nv->cubin(prog, bin.data());
  nv->destroy(&prog);
  cudaFree(nullptr);  // the runtime's context is current on this thread
  CUmodule mod = nullptr;
  CUfunction f = nullptr;
  if (dr->load(&mod, bin.data()) != CUDA_SUCCESS || dr->get(&f, mod, name) != CUDA_SUCCESS)
    return PSB_ERR_UNSUPPORTED;
  if (smem_bytes > 0 &&
      (dr->set_attr(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, smem_bytes) !=
           CUDA_SUCCESS ||
       dr->set_attr(f, CU_FUNC_ATTRIBUTE_PREFERRED_SHARED_MEMORY_CARVEOUT, 100) != CUDA_SUCCESS))
    return PSB_ERR_UNSUPPORTED;
  g_cache[ckey] = f;
  if (__ps_trace) fprintf(__ps_trace, "physis_b200: compiled %s for %s\n", name, key.c_str());
  *fn = f;
  return PSB_OK;
}

psb_status rtc_cached(const std::string &key, CUfunction *fn) {
  *fn = nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PSB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(std::to_string(dev) + "|" + key);
  if (it == g_cache.end() || !it->second) return PSB_ERR_UNSUPPORTED;
  *fn = it->second;
  return PSB_OK;
}

psb_status rtc_launch(CUfunction fn, unsigned blocks, unsigned threads, unsigned smem,
                      cudaStream_t s, void **args) {
  const DriverApi *dr = driver_api();
  if (!dr) return PSB_ERR_UNSUPPORTED;
  const CUresult e = dr->launch(fn, blocks, 1, 1, threads, 1, 1, smem, (CUstream)s, args, nullptr);
  return e == CUDA_SUCCESS ? PSB_OK : set_status(PSB_ERR_CUDA);
}

}  // namespace psb
