// Full FP64 solve that never allocates device memory.
//
// Some callers cannot let a library call cudaMalloc: host frameworks that own all
// device memory through their own pool (and forbid other libraries from carving
// pieces out of it), applications that pre-allocate every byte under a fixed memory
// budget, and latency-sensitive loops that cannot afford the device-wide
// synchronisation cudaMalloc and cudaFree imply.  This entry point serves them: the
// per-pair scratch of the stage kernels (the reduced tile, the tridiagonal, the QL
// rotation log) lives in one fixed array compiled into the library, sized
// SBG_NOALLOC_SCRATCH_BYTES.  Every GPU that loads the library holds that array
// until the process exits.
//
// Rules the implementation follows:
//   * host code never hands the array's name to a kernel (on the host it is only a
//     stand-in symbol, not a device address); the device address comes from
//     cudaGetSymbolAddress, taken once per device with that device current and cached
//     (so cudaDeviceReset of that device after the first call is not supported: the
//     array moves with the new context and the cached address would dangle);
//   * nothing in the scratch has to start at zero: every stage writes what the next
//     one reads for every pair of the call, so the previous call's leftovers are
//     harmless;
//   * all calls share the one array, so calls that overlap on the GPU (different
//     streams, or different host threads without ordering) race on it.
#include "sbg/geneig.h"
#include "kernels.cuh"
#include "tuning.h"

#include <cstdio>
#include <map>
#include <mutex>
#include <string>

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SBG_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array on the current device (set-up on first use).
cudaError_t scratch_address(void** out) {
    static std::mutex mu;
    static std::map<int, void*> cache;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) { *out = it->second; return cudaSuccess; }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    cache[dev] = p;
    *out = p;
    return cudaSuccess;
}

// Bytes of scratch a batch needs: exactly what carve_workspace spans.
size_t scratch_needed(int n, int batch) { return sbg::workspace_bytes(n, batch); }

// Largest batch of order n the fixed array holds.
size_t max_pairs(int n) {
    size_t p = (static_cast<size_t>(SBG_NOALLOC_SCRATCH_BYTES) - 7 * 256) / sbg::workspace_bytes_per_pair(n);
    while (scratch_needed(n, static_cast<int>(p + 1)) <= static_cast<size_t>(SBG_NOALLOC_SCRATCH_BYTES)) ++p;
    return p;
}

int fail(int status, const std::string& msg) {
    sbg::set_last_error(msg);
    std::fprintf(stderr, "[sbg noalloc] %s\n", msg.c_str());
    return status;
}

}  // namespace

extern "C" int sbg_geneig_full_noalloc_launch(int n, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B,
                                              double* d_W, cuDoubleComplex* d_X, int* d_info, int batch,
                                              cudaStream_t stream) {
    if (n < 1) return fail(SBG_ERR_INVALID_VALUE, "n must be >= 1");
    if (batch < 0) return fail(SBG_ERR_INVALID_VALUE, "batch must be >= 0");
    if (batch == 0) return SBG_OK;
    if (!d_A || !d_B || !d_W || !d_X || !d_info) return fail(SBG_ERR_INVALID_VALUE, "null device pointer");
    if (n > sbg_max_n(SBG_PRECISION_FP64))
        return fail(SBG_ERR_UNSUPPORTED, "n = " + std::to_string(n) + " exceeds the supported maximum");
    const size_t need = scratch_needed(n, batch);
    if (need > static_cast<size_t>(SBG_NOALLOC_SCRATCH_BYTES)) {
        return fail(SBG_ERR_INVALID_VALUE,
                    "batch " + std::to_string(batch) + " at n = " + std::to_string(n) + " needs " +
                        std::to_string(need) + " bytes of scratch; the fixed no-allocation scratch holds " +
                        std::to_string(SBG_NOALLOC_SCRATCH_BYTES) + " bytes, i.e. at most " +
                        std::to_string(max_pairs(n)) + " pairs at this n (split the batch)");
    }
    void* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) return fail(SBG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    const sbg::Workspace ws = sbg::carve_workspace(base, n, batch);
    const sbg::Schedule sch = sbg::default_schedule(n, SBG_PRECISION_FP64);
    const double2* A = reinterpret_cast<const double2*>(d_A);
    const double2* B = reinterpret_cast<const double2*>(d_B);
    double2* X = reinterpret_cast<double2*>(d_X);
    e = sbg::launch_reduce(sbg::kReduceFull, A, B, n, batch, ws, X, d_info, sch.shape(), stream);
    if (e == cudaSuccess) e = sbg::launch_hetrd(n, batch, X, ws, d_info, sch.shape(), stream);
    if (e == cudaSuccess)
        e = sbg::launch_ql_logged(n, batch, ws, d_W, X, d_info, false, sch.chain_threads, sch.ql_warps, stream);
    if (e == cudaSuccess) e = sbg::launch_back(sbg::kBackFull, n, batch, ws, X, d_info, sch.shape(), stream);
    if (e != cudaSuccess) return fail(SBG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return SBG_OK;
}
