// Energy export that allocates nothing: the fixed-point to double conversion of
// kExportEnergies (transfers.cu), writing into a fixed scratch array compiled into the library
// instead of a synthesis' staging buffer, so it works on any STORMM-format energy array in
// device memory, with or without a synthesis handle.
//
// Meant for callers that must not allocate device memory at the point where they read energies:
// a reporting step inside a running minimization or serving loop whose device memory is fully
// committed to the molecules in flight (an HBM admission budget leaves no room for a staging
// buffer, and allocating there can stall the work already queued), or a STORMM ScoreCard
// integrated through the shim, which owns its own device accumulators but no stormm_b200
// synthesis.
//
// The scratch holds kScratchValues doubles (512 KiB).  The first call on each device looks up
// its address with cudaGetSymbolAddress while that device is current and keeps it, with the
// CUDA context it belongs to, for later calls; a call made in another context (the device was
// reset, or the caller made a context of its own current) looks the address up again, since
// the module holding the array is loaded anew in every context.  Nothing in the scratch needs
// to start at zero: every value a call reads back was written by that call's kernel.  All calls
// on one device share the one array, so calls that overlap in time (different streams or host
// threads) race on it; order them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "stormm_b200.h"
#include "synthesis.h"

namespace sb {

cudaError_t launchExportEnergies(const unsigned long long* nrg, int n, double inv_scale,
                                 double* d_out, cudaStream_t stream);

namespace {

constexpr int kScratchValues = 65536;     // 4,096 systems x 16 energy slots
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_energy_scratch[kScratchValues];

std::mutex g_scratch_mutex;
double* g_scratch_address[kMaxDevices] = {};
CUcontext g_scratch_context[kMaxDevices] = {};

// The calling thread's current CUDA context (null before the runtime has made one current),
// through the driver's cuCtxGetCurrent as the runtime hands it out, so that the library needs
// no link to the driver library
CUcontext currentContext() {
  using CtxGetCurrent = CUresult (*)(CUcontext*);
  static const CtxGetCurrent get = []() -> CtxGetCurrent {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) !=
        cudaSuccess || found != cudaDriverEntryPointSuccess) {
      return nullptr;
    }
    return reinterpret_cast<CtxGetCurrent>(fn);
  }();
  if (get == nullptr) {
    throw Error(SB_ERR_CUDA, "cuCtxGetCurrent is not available from the CUDA runtime");
  }
  CUcontext ctx = nullptr;
  if (get(&ctx) != CUDA_SUCCESS) {
    throw Error(SB_ERR_CUDA, "cuCtxGetCurrent failed");
  }
  return ctx;
}

// Address of this device's scratch in the current context: looked up once per device and
// context, with that device current
double* scratchAddress(int device) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  const CUcontext ctx = currentContext();
  if (g_scratch_address[device] == nullptr || ctx == nullptr ||
      ctx != g_scratch_context[device]) {
    void* p = nullptr;
    cudaCheck(cudaGetSymbolAddress(&p, g_energy_scratch), "cudaGetSymbolAddress(energy scratch)");
    g_scratch_address[device] = static_cast<double*>(p);
    g_scratch_context[device] = currentContext();   // current now, if it was not before
  }
  return g_scratch_address[device];
}

}  // namespace

}  // namespace sb

extern "C" int sb_energies_to_host_static(const int64_t* d_energies, int nsys, int stride,
                                          int nrg_bits, double* energies, void* stream) {
  try {
    if (nsys < 0 || stride <= 0 || nrg_bits < 0 || nrg_bits > 62) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_energies_to_host_static: bad system count, stride "
                      "or fixed-point bits");
    }
    const long long n = static_cast<long long>(nsys) * stride;
    if (n > sb::kScratchValues) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_energies_to_host_static: " + std::to_string(n) +
                      " values exceed the static scratch of " +
                      std::to_string(sb::kScratchValues) + " doubles (4,096 systems of 16 "
                      "slots); use sb_get_energies for larger syntheses");
    }
    int device = 0;
    sb::cudaCheck(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= sb::kMaxDevices) {
      throw sb::Error(SB_ERR_DEVICE, "sb_energies_to_host_static: device ordinal out of range");
    }
    double* scratch = sb::scratchAddress(device);
    if (n == 0) {
      return SB_OK;   // set-up only
    }
    if (d_energies == nullptr || energies == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_energies_to_host_static: null array");
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    sb::cudaCheck(sb::launchExportEnergies(reinterpret_cast<const unsigned long long*>(d_energies),
                                           static_cast<int>(n), std::ldexp(1.0, -nrg_bits),
                                           scratch, s), "energy conversion");
    sb::cudaCheck(cudaMemcpyAsync(energies, scratch, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                  s), "energy download");
    sb::cudaCheck(cudaStreamSynchronize(s), "energy download");
    return SB_OK;
  }
  catch (const sb::Error &e) {
    sb::setLastError(e.what());
    return e.code;
  }
  catch (const std::exception &e) {
    sb::setLastError(e.what());
    return SB_ERR_ARGUMENT;
  }
}
