// Internal: the solver handle behind the C ABI (capi.cu) and the uneven-n queue
// (queue.cu), with the error plumbing both use.  Not part of the public header.
#pragma once

#include "sbg/geneig.h"
#include "kernels.cuh"
#include "tuning.h"

#include <cuda.h>        // driver types only: cuPointerGetAttribute is reached through the runtime

#include <algorithm>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace sbgi {

extern thread_local std::string g_last_error;

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(e == cudaErrorMemoryAllocation ? SBG_ERR_NO_MEMORY : SBG_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return SBG_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return SBG_ERR_INTERNAL;
    } catch (...) {
        g_last_error = "unknown exception";
        return SBG_ERR_INTERNAL;
    }
}

// Device workspace of one stream slot; grows on demand, never during capture.
struct Slot {
    void* ptr = nullptr;
    size_t bytes = 0;
    int capacity = 0;
};

inline int default_chunk_pairs(int n, bool mixed = false) {
    const size_t per = sbg::workspace_bytes_per_pair(n, mixed);
    const size_t target = size_t(1) << 30;     // about 1 GiB of scratch per stream slot
    size_t pairs = target / std::max<size_t>(per, 1);
    pairs = std::min<size_t>(std::max<size_t>(pairs, 1024), 65536);
    return static_cast<int>(pairs);
}


struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) check_cuda(cudaSetDevice(dev), "cudaSetDevice");
    }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// Device-side address of the host range [p, p + bytes) when one pinned, device-mapped allocation
// holds all of it (so a kernel may read every byte of it), else nullptr.  Both ends must be
// mapped host memory of the same allocation (the driver's buffer id), at the same distance on
// the device side; any failed query means "no".
inline const void* mapped_host_range(const void* p, size_t bytes) {
    if (!p || bytes == 0) return nullptr;
    using AttrFn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
    static const AttrFn attr = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<AttrFn>(nullptr);
        }
        return reinterpret_cast<AttrFn>(f);
    }();
    if (!attr) return nullptr;
    const char* lo = static_cast<const char*>(p);
    const char* hi = lo + bytes - 1;
    cudaPointerAttributes a{}, b{};
    if (cudaPointerGetAttributes(&a, lo) != cudaSuccess || cudaPointerGetAttributes(&b, hi) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
        return nullptr;
    if (static_cast<const char*>(b.devicePointer) - static_cast<const char*>(a.devicePointer) !=
        static_cast<ptrdiff_t>(bytes - 1))
        return nullptr;
    unsigned long long id_lo = 0, id_hi = 1;
    if (attr(&id_lo, CU_POINTER_ATTRIBUTE_BUFFER_ID, reinterpret_cast<CUdeviceptr>(lo)) != CUDA_SUCCESS ||
        attr(&id_hi, CU_POINTER_ATTRIBUTE_BUFFER_ID, reinterpret_cast<CUdeviceptr>(hi)) != CUDA_SUCCESS ||
        id_lo != id_hi)
        return nullptr;
    return a.devicePointer;
}

// Creates a solver for order n (throws Error).
void create_solver(int n, int device, const sbg_solver_options* o, sbg_solver** out);

}  // namespace sbgi

using namespace sbgi;

struct sbg_solver {
    int n = 0;
    int device = 0;
    int precision = SBG_PRECISION_FP64;
    int refine_steps = 5;
    int chunk_pairs = 0;
    unsigned long long* d_redo = nullptr;   // mixed form: pairs handed to the FP64 re-solve
    sbg::Schedule sched;
    bool autotuned = false;
    bool sweep_ran = false;
    const char* layer = "compile";
    std::mutex mu;
    std::vector<Slot> slots;
    // Workspace slot i serves stream slot_streams[i]: launches on different streams never share
    // scratch (the reference's launches keep everything in shared memory, so they are independent
    // across streams, and so are these).  The first stream a solver sees gets slot 0.
    std::vector<cudaStream_t> slot_streams;
    // staging buffers of the host-buffer path, one per internal stream
    // (pull: a high-priority stream for the kernel that reads B's lower triangle from mapped host
    // memory; pulled / consumed order it against the chunk's own stream.)
    struct Staging { void* A = nullptr; void* B = nullptr; void* X = nullptr; void* W = nullptr; void* info = nullptr;
                     int capacity = 0; cudaStream_t stream = nullptr; cudaStream_t pull = nullptr;
                     cudaEvent_t pulled = nullptr; cudaEvent_t consumed = nullptr; };
    std::vector<Staging> staging;
    std::mutex host_mu;                 // one solve_host at a time: they share the staging buffers
    // bytes the last solve_host moved over the host link, each way
    long long last_h2d_bytes = 0, last_d2h_bytes = 0;
    // per-stage event timing
    bool timing = false;
    struct StageEvents { int stage; int kernels; cudaEvent_t a, b; };
    std::vector<StageEvents> stage_events;

    ~sbg_solver() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        for (auto& s : slots) if (s.ptr) cudaFree(s.ptr);
        if (d_redo) cudaFree(d_redo);
        for (auto& st : staging) {
            if (st.stream) cudaStreamDestroy(st.stream);
            if (st.pull) cudaStreamDestroy(st.pull);
            if (st.pulled) cudaEventDestroy(st.pulled);
            if (st.consumed) cudaEventDestroy(st.consumed);
            for (void* p : {st.A, st.B, st.X, st.W, st.info}) if (p) cudaFree(p);
        }
        for (auto& e : stage_events) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
        cudaSetDevice(prev);
    }

    void stage_begin(cudaStream_t stream, cudaEvent_t* a) {
        *a = nullptr;
        if (!timing) return;
        check_cuda(cudaEventCreate(a), "cudaEventCreate");
        check_cuda(cudaEventRecord(*a, stream), "cudaEventRecord");
    }
    void stage_end(cudaStream_t stream, cudaEvent_t a, int stage, int kernels) {
        if (!timing || !a) return;
        cudaEvent_t b;
        check_cuda(cudaEventCreate(&b), "cudaEventCreate");
        check_cuda(cudaEventRecord(b, stream), "cudaEventRecord");
        std::lock_guard<std::mutex> lock(mu);
        stage_events.push_back({stage, kernels, a, b});
    }

    int slot_for(cudaStream_t st) {
        std::lock_guard<std::mutex> lock(mu);
        for (size_t i = 0; i < slot_streams.size(); ++i)
            if (slot_streams[i] == st) return static_cast<int>(i);
        slot_streams.push_back(st);
        return static_cast<int>(slot_streams.size()) - 1;
    }

    sbg::Workspace workspace(int slot_idx, int pairs, cudaStream_t stream) {
        std::lock_guard<std::mutex> lock(mu);
        if (static_cast<int>(slots.size()) <= slot_idx) slots.resize(slot_idx + 1);
        Slot& s = slots[slot_idx];
        if (s.capacity < pairs) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (stream) check_cuda(cudaStreamIsCapturing(stream, &cs), "cudaStreamIsCapturing");
            if (cs != cudaStreamCaptureStatusNone)
                throw Error(SBG_ERR_CAPTURING, "workspace must grow while the stream is capturing; "
                                               "call sbg_solver_reserve before capture");
            if (s.ptr) { check_cuda(cudaFree(s.ptr), "cudaFree"); s.ptr = nullptr; s.capacity = 0; }
            const size_t bytes = sbg::workspace_bytes(n, pairs, precision == SBG_PRECISION_MIXED);
            check_cuda(cudaMalloc(&s.ptr, bytes), "cudaMalloc(workspace)");
            s.bytes = bytes;
            s.capacity = pairs;
        }
        sbg::Workspace w = sbg::carve_workspace(s.ptr, n, s.capacity, precision == SBG_PRECISION_MIXED);
        if (precision == SBG_PRECISION_MIXED) {
            if (!d_redo) {
                check_cuda(cudaMalloc(&d_redo, sizeof(unsigned long long)), "cudaMalloc(redo counter)");
                check_cuda(cudaMemset(d_redo, 0, sizeof(unsigned long long)), "cudaMemset(redo counter)");
            }
            w.redo_count = d_redo;
        }
        return w;
    }

    // The mixed form above kMixedMaxN: FP64 reduction, complex64 Householder (one CTA per pair),
    // FP64 eigenpairs of that T and Y = Q Z, the FP64 refinement on the pair's matrices in the
    // workspace, X = L^{-H} Y for the pairs it converged; then the pairs it gave up on (ws.rstat ==
    // kRefineRedo) are solved again by the FP64 stage kernels, every other pair left untouched.
    void run_chunk_mixed_big(const double2* A, const double2* B, double* W, double2* X, int* info, int cnt,
                             const sbg::Workspace& ws, cudaStream_t stream) {
        cudaEvent_t ev;
        stage_begin(stream, &ev);
        check_cuda(sbg::launch_reduce(sbg::kReduceMixed, A, B, n, cnt, ws, X, info, sched.shape(), stream),
                   "reduce kernel");
        stage_end(stream, ev, 0, 1);
        stage_begin(stream, &ev);
        check_cuda(sbg::launch_hetrd_c64_big(n, cnt, X, ws, info, stream), "complex64 hetrd kernel");
        stage_end(stream, ev, 1, 1);
        stage_begin(stream, &ev);
        check_cuda(sbg::launch_ql_logged(n, cnt, ws, W, X, info, false, sched.chain_threads, sched.ql_warps, stream),
                   "QL kernels");
        check_cuda(sbg::launch_back(sbg::kBackQOnly, n, cnt, ws, X, info, sched.shape(), stream), "Q-apply kernel");
        check_cuda(sbg::launch_refine_big(n, cnt, ws, W, X, info, refine_steps, stream), "refinement kernel");
        stage_end(stream, ev, 2, sbg::eig_kernel_count(n, false) + 2);
        stage_begin(stream, &ev);
        sbg::Workspace sel = ws;
        sel.sel = ws.rstat;
        sel.sel_mask = (1 << sbg::kRefineDone) | (1 << sbg::kRefineSkip);
        check_cuda(sbg::launch_back(sbg::kBackLOnly, n, cnt, sel, X, info, sched.shape(), stream),
                   "back-transform kernel");
        sel.sel_mask = 1 << sbg::kRefineRedo;                   // the FP64 solve of the pairs left over
        check_cuda(sbg::launch_reduce(sbg::kReduceFull, A, B, n, cnt, sel, X, info, sched.shape(), stream),
                   "reduce kernel (FP64 redo)");
        check_cuda(sbg::launch_hetrd(n, cnt, X, sel, info, sched.shape(), stream), "hetrd kernel (FP64 redo)");
        check_cuda(sbg::launch_ql_logged(n, cnt, sel, W, X, info, false, sched.chain_threads, sched.ql_warps, stream),
                   "QL kernels (FP64 redo)");
        check_cuda(sbg::launch_back(sbg::kBackFull, n, cnt, sel, X, info, sched.shape(), stream),
                   "back-transform kernel (FP64 redo)");
        stage_end(stream, ev, 3, 1 + 1 + (n > sbg::kSmallMaxN ? 0 : 1) + sbg::eig_kernel_count(n, false) + 1);
    }

    // One chunk of at most chunk_pairs pairs through the three stages.
    void run_chunk(const double2* A, const double2* B, double* W, double2* X, int* info, int cnt,
                   const sbg::Workspace& ws, cudaStream_t stream) {
        if (sbg::mixed_big(n, precision == SBG_PRECISION_MIXED)) {
            run_chunk_mixed_big(A, B, W, X, info, cnt, ws, stream);
            return;
        }
        cudaEvent_t ev;
        stage_begin(stream, &ev);
        check_cuda(sbg::launch_reduce(sbg::kReduceFull, A, B, n, cnt, ws, X, info, sched.shape(), stream),
                   "reduce kernel");
        stage_end(stream, ev, 0, sbg::reduce_kernel_count(n, sched.reduce_tc != 0));
        const bool mixed = precision == SBG_PRECISION_MIXED;
        stage_begin(stream, &ev);
        if (mixed)
            check_cuda(sbg::launch_hetrd_c64(n, cnt, X, ws, info, sched.shape(), stream), "complex64 hetrd kernel");
        else
            check_cuda(sbg::launch_hetrd(n, cnt, X, ws, info, sched.shape(), stream), "hetrd kernel");
        stage_end(stream, ev, 1, n > sbg::kSmallMaxN ? 0 : 1);       // large n: inside the reduce kernel
        stage_begin(stream, &ev);
        if (mixed)             // eigenpairs of the complex64 T, Y = Q Z, FP64 refinement against C
            check_cuda(sbg::launch_eig_mixed(n, cnt, ws, W, X, info, refine_steps, sched.chain_threads, sched.shape(),
                                             stream),
                       "mixed eigensolve kernels");
        else
            check_cuda(sbg::launch_ql_logged(n, cnt, ws, W, X, info, false, sched.chain_threads, sched.ql_warps,
                                             stream), "QL kernels");
        stage_end(stream, ev, 2, sbg::eig_kernel_count(n, mixed));
        stage_begin(stream, &ev);
        check_cuda(sbg::launch_back(mixed ? sbg::kBackLOnly : sbg::kBackFull, n, cnt, ws, X, info, sched.shape(),
                                    stream), "back-transform kernel");
        stage_end(stream, ev, 3, !mixed && n > 56 && sched.reduce_tc ? 2 : 1);
    }

    // Host buffers in, host buffers out, chunks round-robin over nstreams internal streams.  A goes
    // through the copy engine; B, of which only the lower triangle is ever read, is pulled by a
    // kernel when the caller's buffer is pinned and device-mapped (25 % fewer bytes over the host
    // link at n = 54), else copied whole.
    void solve_host(const double2* hA, const double2* hB, double* hW, double2* hX, int* hinfo, int batch,
                    int chunk, int nstreams) {
        if (batch < 0 || chunk <= 0 || nstreams <= 0) throw Error(SBG_ERR_INVALID_VALUE, "bad solve_host arguments");
        std::lock_guard<std::mutex> serial(host_mu);
        last_h2d_bytes = last_d2h_bytes = 0;
        if (batch == 0) return;
        if (!hA || !hB || !hW || !hX || !hinfo) throw Error(SBG_ERR_INVALID_VALUE, "null host pointer");
        chunk = std::min(chunk, batch);
        const size_t nn = static_cast<size_t>(n) * n;
        const double2* dB_host =
            static_cast<const double2*>(mapped_host_range(hB, 16 * nn * static_cast<size_t>(batch)));
        {
            std::lock_guard<std::mutex> lock(mu);
            if (static_cast<int>(staging.size()) < nstreams) staging.resize(nstreams);
            int lo_prio = 0, hi_prio = 0;
            check_cuda(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio), "cudaDeviceGetStreamPriorityRange");
            for (int i = 0; i < nstreams; ++i) {
                Staging& st = staging[i];
                if (!st.stream) check_cuda(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking), "cudaStreamCreate");
                if (!st.pull)
                    check_cuda(cudaStreamCreateWithPriority(&st.pull, cudaStreamNonBlocking, hi_prio),
                               "cudaStreamCreateWithPriority");
                if (!st.pulled) check_cuda(cudaEventCreateWithFlags(&st.pulled, cudaEventDisableTiming), "cudaEventCreate");
                if (!st.consumed)
                    check_cuda(cudaEventCreateWithFlags(&st.consumed, cudaEventDisableTiming), "cudaEventCreate");
                if (st.capacity < chunk) {
                    for (void** p : {&st.A, &st.B, &st.X, &st.W, &st.info}) if (*p) { cudaFree(*p); *p = nullptr; }
                    check_cuda(cudaMalloc(&st.A, 16 * nn * chunk), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.B, 16 * nn * chunk), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.X, 16 * nn * chunk), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.W, 8 * static_cast<size_t>(n) * chunk), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.info, 4 * static_cast<size_t>(chunk)), "cudaMalloc(staging)");
                    st.capacity = chunk;
                }
            }
        }
        const size_t lower_bytes = 8 * static_cast<size_t>(n) * (n + 1);      // rows j..n-1 of every column j
        int idx = 0;
        for (int off = 0; off < batch; off += chunk, ++idx) {
            const int cnt = std::min(chunk, batch - off);
            Staging& st = staging[idx % nstreams];
            check_cuda(cudaMemcpyAsync(st.A, hA + nn * off, 16 * nn * cnt, cudaMemcpyHostToDevice, st.stream), "H2D A");
            if (dB_host) {
                // the previous chunk of this slot has finished reading its B once `consumed` fires
                check_cuda(cudaStreamWaitEvent(st.pull, st.consumed, 0), "cudaStreamWaitEvent");
                check_cuda(sbg::launch_pull_pairs(dB_host + nn * off, static_cast<double2*>(st.B), cnt, n, true,
                                                  st.pull), "host pull kernel");
                check_cuda(cudaEventRecord(st.pulled, st.pull), "cudaEventRecord");
                check_cuda(cudaStreamWaitEvent(st.stream, st.pulled, 0), "cudaStreamWaitEvent");
                last_h2d_bytes += static_cast<long long>(lower_bytes) * cnt;
            } else {
                check_cuda(cudaMemcpyAsync(st.B, hB + nn * off, 16 * nn * cnt, cudaMemcpyHostToDevice, st.stream),
                           "H2D B");
                last_h2d_bytes += static_cast<long long>(16 * nn) * cnt;
            }
            last_h2d_bytes += static_cast<long long>(16 * nn) * cnt;
            launch(static_cast<double2*>(st.A), static_cast<double2*>(st.B), static_cast<double*>(st.W),
                   static_cast<double2*>(st.X), static_cast<int*>(st.info), cnt, st.stream);
            check_cuda(cudaEventRecord(st.consumed, st.stream), "cudaEventRecord");
            check_cuda(cudaMemcpyAsync(hX + nn * off, st.X, 16 * nn * cnt, cudaMemcpyDeviceToHost, st.stream), "D2H X");
            check_cuda(cudaMemcpyAsync(hW + static_cast<size_t>(n) * off, st.W, 8 * static_cast<size_t>(n) * cnt,
                                       cudaMemcpyDeviceToHost, st.stream), "D2H W");
            check_cuda(cudaMemcpyAsync(hinfo + off, st.info, 4 * static_cast<size_t>(cnt), cudaMemcpyDeviceToHost,
                                       st.stream), "D2H info");
            last_d2h_bytes += static_cast<long long>(16 * nn + 8 * n + 4) * cnt;
        }
        for (int i = 0; i < nstreams; ++i) check_cuda(cudaStreamSynchronize(staging[i].stream), "cudaStreamSynchronize");
    }

    void launch(const double2* A, const double2* B, double* W, double2* X, int* info, int batch,
                cudaStream_t stream, int slot_idx = -1) {
        if (batch < 0) throw Error(SBG_ERR_INVALID_VALUE, "batch < 0");
        if (batch == 0) return;
        if (!A || !B || !W || !X || !info) throw Error(SBG_ERR_INVALID_VALUE, "null device pointer");
        const size_t nn = static_cast<size_t>(n) * n;
        const int cap = std::min(batch, chunk_pairs);
        if (slot_idx < 0) slot_idx = slot_for(stream);
        sbg::Workspace ws = workspace(slot_idx, cap, stream);
        for (int off = 0; off < batch; off += ws.capacity) {
            const int cnt = std::min(ws.capacity, batch - off);
            run_chunk(A + nn * off, B + nn * off, W + static_cast<size_t>(n) * off, X + nn * off, info + off,
                      cnt, ws, stream);
        }
    }
};
