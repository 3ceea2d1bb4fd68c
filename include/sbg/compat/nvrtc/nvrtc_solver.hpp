// Drop-in for the runtime-n solver header of riteshbhirud/sunny-batched-geneig
// (src/nvrtc/nvrtc_solver.hpp).  It has the same public API: NvrtcGeneigSolver, TuningMode,
// CacheMode, ModuleCacheKey, make_streams and destroy_streams.  It is header-only, written over the
// C ABI of sbg/geneig.h.
//
// A caller written against the reference, which does
//     #include "nvrtc/nvrtc_solver.hpp"
// compiles unchanged with -I<repo>/include/sbg/compat -I<repo>/include. Link it against
// libsbg_geneig.so and the CUDA driver library (-lcuda).
//
// What differs from the reference, by design (every kernel is compiled ahead of time for sm_100a):
//  * Construction selects a schedule instead of JIT-compiling a kernel.
//    - cache_layer_used() says where the schedule came from: "in-process", "disk" (the
//      checksummed autotune table), or "compile". "compile" is the reference's name for "produced
//      by this construction": the built-in schedule, or a fresh autotune sweep.
//    - cubin_path() names the autotune table of the current device. That is the on-disk artefact
//      of the cache, and one table holds every key.
//  * batches_per_block, block_dim and force_block_dim_x describe the launch shapes this library
//    actually uses (sbg/geneig.h, sbg_solver_options).
//    - A request it cannot honour throws from the constructor, as the reference's does for a
//      BPB that does not fit.
//  * launch() accepts any batch_size >= 0. The reference's partial last block was unchecked.
#pragma once

#include <cuda.h>
#include <vector_types.h>  // dim3

#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include <sbg/geneig.h>

namespace sbg_compat {

[[noreturn]] inline void throw_cu(CUresult r, const char* call) {
    const char* msg = nullptr;
    cuGetErrorString(r, &msg);
    throw std::runtime_error(std::string(call) + " failed: " + (msg ? msg : "unknown CUDA driver error"));
}

inline void check_cu(CUresult r, const char* call) {
    if (r != CUDA_SUCCESS) throw_cu(r, call);
}

[[noreturn]] inline void throw_sbg(int status, const char* call) {
    throw std::runtime_error(std::string(call) + " failed: " + sbg_status_string(status) + ": " + sbg_last_error());
}

inline std::string table_path_of_current_device() {
    CUdevice dev = 0;
    if (cuCtxGetDevice(&dev) != CUDA_SUCCESS) dev = 0;       // no current context: device 0
    char buf[4096];
    const int st = sbg_tuning_table_path(static_cast<int>(dev), buf, sizeof buf);
    if (st != SBG_OK) throw_sbg(st, "sbg_tuning_table_path");
    return std::string(buf);
}

}  // namespace sbg_compat

// nvrtc_solver.hpp:29-30: streams created non-blocking, destroyed and cleared.
inline std::vector<CUstream> make_streams(int n) {
    std::vector<CUstream> v;
    v.reserve(n > 0 ? n : 0);
    for (int i = 0; i < n; ++i) {
        CUstream s = nullptr;
        sbg_compat::check_cu(cuStreamCreate(&s, CU_STREAM_NON_BLOCKING), "cuStreamCreate");
        v.push_back(s);
    }
    return v;
}

inline void destroy_streams(std::vector<CUstream>& streams) {
    for (CUstream s : streams)
        if (s) cuStreamDestroy(s);
    streams.clear();
}

enum class TuningMode { Suggested, Autotune };          // nvrtc_solver.hpp:38
enum class CacheMode { Auto, NoDisk, NoCache };         // nvrtc_solver.hpp:46

// nvrtc_solver.hpp:70-81.  Kept for callers that build keys, e.g. to name the cache file.
struct ModuleCacheKey {
    int n = 0;
    int bpb = 0;
    int arch = 0;
    int block_dim_x = 0;
    bool operator<(const ModuleCacheKey& o) const {
        return std::tie(n, bpb, arch, block_dim_x) < std::tie(o.n, o.bpb, o.arch, o.block_dim_x);
    }
};

class NvrtcGeneigSolver {
public:
    // nvrtc_solver.hpp:99-105.  Like the reference's constructor (nvrtc_solver.cpp:938-939) it
    // retains the device's primary context and makes it current, so buffers the caller then
    // allocates with cuMemAlloc live in the context the library's kernels run in.
    explicit NvrtcGeneigSolver(int n, int device_id, int batches_per_block_request = 0, int force_block_dim_x = 0,
                               TuningMode tuning_mode = TuningMode::Suggested,
                               CacheMode cache_mode = CacheMode::Auto)
        : n_(n) {
        sbg_compat::check_cu(cuInit(0), "cuInit");
        sbg_compat::check_cu(cuDeviceGet(&device_, device_id), "cuDeviceGet");
        sbg_compat::check_cu(cuDevicePrimaryCtxRetain(&context_, device_), "cuDevicePrimaryCtxRetain");
        const CUresult set = cuCtxSetCurrent(context_);
        if (set != CUDA_SUCCESS) {
            cuDevicePrimaryCtxRelease(device_);
            sbg_compat::throw_cu(set, "cuCtxSetCurrent");
        }
        sbg_solver_options o;
        sbg_solver_options_init(&o);
        o.batches_per_block = batches_per_block_request > 0 ? batches_per_block_request : 0;
        o.force_block_dim_x = force_block_dim_x > 0 ? force_block_dim_x : 0;
        o.tuning_mode = tuning_mode == TuningMode::Autotune ? SBG_TUNING_AUTOTUNE : SBG_TUNING_SUGGESTED;
        o.cache_mode = cache_mode == CacheMode::Auto     ? SBG_CACHE_AUTO
                       : cache_mode == CacheMode::NoDisk ? SBG_CACHE_NO_DISK
                                                         : SBG_CACHE_NONE;
        const auto t0 = std::chrono::steady_clock::now();
        const int st = sbg_solver_create(n, device_id, &o, &s_);
        acquire_module_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (st != SBG_OK) {
            cuDevicePrimaryCtxRelease(device_);
            sbg_compat::throw_sbg(st, "NvrtcGeneigSolver");
        }
        const std::string layer = sbg_solver_cache_layer_used(s_);
        cache_layer_used_ = (layer == "in-process") ? "in-process" : (layer == "disk") ? "disk" : "compile";
    }

    ~NvrtcGeneigSolver() {
        sbg_solver_destroy(s_);
        cuDevicePrimaryCtxRelease(device_);
    }

    NvrtcGeneigSolver(const NvrtcGeneigSolver&) = delete;
    NvrtcGeneigSolver& operator=(const NvrtcGeneigSolver&) = delete;
    NvrtcGeneigSolver(NvrtcGeneigSolver&&) = delete;
    NvrtcGeneigSolver& operator=(NvrtcGeneigSolver&&) = delete;

    // nvrtc_solver.hpp:113-115: H x = lambda S x for batch_size column-major pairs; W ascending,
    // U the S-orthonormal eigenvectors, info per pair (zhegv's codes).
    void launch(CUdeviceptr d_H, CUdeviceptr d_S, CUdeviceptr d_W, CUdeviceptr d_U, CUdeviceptr d_info,
                int batch_size, CUstream stream) {
        const int st = sbg_solver_launch(s_, reinterpret_cast<const cuDoubleComplex*>(d_H),
                                         reinterpret_cast<const cuDoubleComplex*>(d_S), reinterpret_cast<double*>(d_W),
                                         reinterpret_cast<cuDoubleComplex*>(d_U), reinterpret_cast<int*>(d_info),
                                         batch_size, stream);
        if (st != SBG_OK) sbg_compat::throw_sbg(st, "NvrtcGeneigSolver::launch");
    }

    // nvrtc_solver.hpp:118-121: chunks of chunk_size pairs round-robin over the first num_streams
    // streams, no synchronisation between them.
    void launch_chunked(CUdeviceptr d_H, CUdeviceptr d_S, CUdeviceptr d_W, CUdeviceptr d_U, CUdeviceptr d_info,
                        int total_matrices, int chunk_size, int num_streams, const std::vector<CUstream>& streams) {
        if (num_streams < 0 || static_cast<size_t>(num_streams) > streams.size())
            throw std::runtime_error("NvrtcGeneigSolver::launch_chunked: num_streams exceeds streams.size()");
        const int st = sbg_solver_launch_chunked(
            s_, reinterpret_cast<const cuDoubleComplex*>(d_H), reinterpret_cast<const cuDoubleComplex*>(d_S),
            reinterpret_cast<double*>(d_W), reinterpret_cast<cuDoubleComplex*>(d_U), reinterpret_cast<int*>(d_info),
            total_matrices, chunk_size, num_streams, streams.data());
        if (st != SBG_OK) sbg_compat::throw_sbg(st, "NvrtcGeneigSolver::launch_chunked");
    }

    int matrix_size() const { return n_; }
    int batches_per_block() const { return sbg_solver_batches_per_block(s_); }
    dim3 block_dim() const { return dim3(static_cast<unsigned>(sbg_solver_block_dim_x(s_)), 1, 1); }
    unsigned int shared_mem_bytes() const { return sbg_solver_shared_mem_bytes(s_); }

    int autotuned_block_dim_x() const { return was_autotuned() ? sbg_solver_block_dim_x(s_) : 0; }
    bool was_autotuned() const { return sbg_solver_was_autotuned(s_) != 0; }
    bool autotune_sweep_ran() const { return sbg_solver_autotune_sweep_ran(s_) != 0; }

    const char* cache_layer_used() const { return cache_layer_used_; }
    double acquire_module_ms() const { return acquire_module_ms_; }

    // The directory of the autotune table: $SUNNY_GENEIG_CACHE_DIR if set (the reference's
    // variable), else $XDG_CACHE_HOME/sunny_geneig_b200, else $HOME/.cache/sunny_geneig_b200.
    static std::string cache_dir() {
        const std::string p = sbg_compat::table_path_of_current_device();
        const size_t slash = p.find_last_of('/');
        return slash == std::string::npos ? std::string(".") : p.substr(0, slash);
    }
    // The autotune table of the current device, which holds the schedules of every key.
    static std::string cubin_path(const ModuleCacheKey&) { return sbg_compat::table_path_of_current_device(); }

private:
    int n_ = 0;
    CUdevice device_ = 0;
    CUcontext context_ = nullptr;
    sbg_solver* s_ = nullptr;
    const char* cache_layer_used_ = "compile";
    double acquire_module_ms_ = 0.0;
};
