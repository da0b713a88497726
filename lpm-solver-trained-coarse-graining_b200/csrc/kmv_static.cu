// K.u without caller-provided scratch: the entry point lpm_kmv_f64_static.
//
// The two-pass operator needs a scratch buffer of 4 values per particle and system (the shell sums S0, S1, TS0, TS1
// that pass 2 reads at the neighbours).  lpm_kmv_sc_f64 / lpm_kmv_sq_f64 take that buffer from the caller.  Some
// callers cannot provide one: they hold device pointers handed to them by someone else but have no device allocator
// of their own (a foreign-language host that only passes pointers through an FFI), or they run where allocating is
// not allowed or not acceptable (inside a fixed memory budget, or on a latency-critical path where a cudaMalloc and
// its implicit synchronisation would stall).  This file serves them from a fixed device array instead.
//
// The array below is a file-scope __device__ variable of LPM_KMV_STATIC_SCRATCH_BYTES.  Every GPU that loads the
// library holds it for the life of the process.  Host code cannot use its name as a device address (on the host the
// name refers to a host-side shadow), so on the first call on each device, with that device current, the device
// address is looked up with cudaGetSymbolAddress and cached; that first call should therefore come before any stream
// capture.  The cached address belongs to the device context it was looked up in: after a cudaDeviceReset (which
// ends that context) it is stale, so a process that resets a device must not call this entry point on it again.
// All calls on a device share the one array: two calls whose work overlaps on that GPU (different streams,
// or several host threads) race on it and must be serialised by the caller.  Pass 1 overwrites every entry that pass 2
// later reads, so the array needs no clearing between calls.  No call allocates or frees device memory.
#include <mutex>

#include "../../include/lpm_b200.h"
#include "lpm_abi.h"
#include "lpm_kernels.h"

namespace {

constexpr size_t kStaticDoubles = LPM_KMV_STATIC_SCRATCH_BYTES / sizeof(double);

static __device__ __align__(256) double g_kmv_scratch[kStaticDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_kmv_scratch on the current device (looked up once per device).
int static_scratch(double** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= kMaxDevices) return LPM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_kmv_scratch);
        if (e != cudaSuccess) return (int)e;
        if (!p) return LPM_ERR_UNSUPPORTED;
        g_addr[dev] = p;
    }
    *out = static_cast<double*>(g_addr[dev]);
    return LPM_OK;
}

}  // namespace

extern "C" int lpm_kmv_f64_static(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv,
                                  int32_t coef_layout, const lpm_batch* batch, double* out, void* stream)
{
    using namespace lpm;
    if (!u || !Kn || !Tv || !out) return LPM_ERR_ARG;
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(coef_layout, L, cl))) return rc;
    // 4 shell sums per particle and system must fit the static array
    const double need = 4.0 * (double)bt.nsys * (double)L.N;
    if (need > (double)kStaticDoubles) return LPM_ERR_WORKSPACE;
    double* scratch = nullptr;
    if ((rc = static_scratch(&scratch)) != LPM_OK) return rc;
    const cudaError_t e =
        launch_kmv<double>(L, u, Kn, Tv, cl, bt, out, scratch, nullptr, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? LPM_OK : (int)e;
}
