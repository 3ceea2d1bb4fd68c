// C ABI of the batched generalized eigensolver: the fixed n = 54 drop-in of
// src/geneig_fixed.cu and the runtime-n solver handle that mirrors
// NvrtcGeneigSolver (src/nvrtc/nvrtc_solver.hpp).  Every entry point catches
// C++ exceptions and maps failures to sbg_status codes; the reference's void
// launchers keep their void signatures and report through sbg_last_error() and
// the CUDA error state.
#include "solver.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace sbgi {
thread_local std::string g_last_error;
}  // namespace sbgi

namespace sbg {
void set_last_error(const std::string& msg) { sbgi::g_last_error = msg; }
}  // namespace sbg


namespace {


int supported_max_n(int precision) {
    const size_t lim = static_cast<size_t>(sbg::max_smem_optin());
    int best = 0;
    const bool single = precision == SBG_PRECISION_MIXED;
    for (int n = 1; n <= sbg::kBigMaxN; ++n) {
        // the mixed form above kMixedMaxN: the FP64 kernels (its own re-solve) plus the complex64
        // Householder (one CTA per pair); the refinement's shared memory is fixed and small
        if (single && n > sbg::kMixedBigMaxN) break;
        const bool big_mixed = single && n > sbg::kMixedMaxN;
        if (n > sbg::kSmallMaxN) {          // cluster kernels
            size_t need = std::max(sbg::big_reduce_smem_bytes(n), sbg::ql_rows_smem_bytes(n, false));
            need = std::max(need, sbg::ql_chain_smem_bytes(n, 32, false));
            if (big_mixed) need = std::max(need, sbg::hetrd_c64_big_smem_bytes(n));
            if (sbg::big_path(n) && need <= lim) best = n;
            continue;
        }
        size_t need = std::max(sbg::reduce_smem_bytes(sbg::kReduceFull, n), sbg::back_smem_bytes(n));
        need = std::max(need, sbg::hetrd_smem_bytes(n, 128));
        need = std::max(need, sbg::ql_apply_smem_bytes(n, 1, false));
        need = std::max(need, sbg::ql_chain_smem_bytes(n, 32, false));
        if (big_mixed) {
            need = std::max(need, sbg::hetrd_c64_big_smem_bytes(n));
        } else if (single) {                // complex64 Householder + FP64 tensor-core refinement
            need = std::max(need, sbg::refine_c_smem_bytes(n));
            need = std::max(need, sbg::mixed_fallback_smem_bytes(n));
            need = std::max(need, sbg::hetrd_c64_smem_bytes(n));
        }
        if (need <= lim) best = n;
    }
    return best;
}

}  // namespace

void sbgi::create_solver(int n, int device, const sbg_solver_options* o, sbg_solver** out) {
    if (!out) throw Error(SBG_ERR_INVALID_VALUE, "out == NULL");
    *out = nullptr;
    sbg_solver_options opts;
    sbg_solver_options_init(&opts);
    if (o) opts = *o;
    if (n < 1) throw Error(SBG_ERR_INVALID_VALUE, "n must be >= 1");
    if (opts.precision != SBG_PRECISION_FP64 && opts.precision != SBG_PRECISION_MIXED)
        throw Error(SBG_ERR_INVALID_VALUE, "unknown precision");
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) throw Error(SBG_ERR_INVALID_VALUE, "device_id out of range");
    DeviceGuard g(device);
    if (n > supported_max_n(opts.precision))
        throw Error(SBG_ERR_UNSUPPORTED, "n = " + std::to_string(n) + " exceeds the supported maximum (" +
                                             std::to_string(supported_max_n(opts.precision)) + ")");
    std::unique_ptr<sbg_solver> s(new sbg_solver);
    s->n = n;
    s->device = device;
    s->precision = opts.precision;
    s->refine_steps = opts.refine_steps > 0 ? opts.refine_steps : 5;
    s->chunk_pairs = opts.workspace_pairs > 0 ? opts.workspace_pairs
                                              : default_chunk_pairs(n, opts.precision == SBG_PRECISION_MIXED);
    sbg::TuneRequest req;
    req.n = n;
    req.device = device;
    req.precision = opts.precision;
    req.force_threads = opts.force_block_dim_x;
    req.force_bpb = opts.batches_per_block;
    req.autotune = opts.tuning_mode == SBG_TUNING_AUTOTUNE;
    req.cache_mode = opts.cache_mode;
    sbg::TuneResult tr = sbg::select_schedule(req);
    s->sched = tr.sched;
    s->autotuned = tr.autotuned;
    s->sweep_ran = tr.sweep_ran;
    s->layer = tr.layer;
    *out = s.release();
}

namespace {

// Process-wide n = 54 FP64 solver per device, used by the fixed-size drop-in.
sbg_solver* default_n54_solver() {
    static std::mutex mu;
    static std::map<int, sbg_solver*> solvers;
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    auto it = solvers.find(dev);
    if (it != solvers.end()) return it->second;
    sbg_solver* s = nullptr;
    create_solver(54, dev, nullptr, &s);
    solvers[dev] = s;       // lives until process exit
    return s;
}

void report_void(int status) {
    if (status != SBG_OK) std::fprintf(stderr, "[sbg] %s\n", g_last_error.c_str());
}

const double2* c2(const cuDoubleComplex* p) { return reinterpret_cast<const double2*>(p); }
double2* c2(cuDoubleComplex* p) { return reinterpret_cast<double2*>(p); }

}  // namespace

extern "C" {

const char* sbg_status_string(int status) {
    switch (status) {
        case SBG_OK: return "ok";
        case SBG_ERR_INVALID_VALUE: return "invalid value";
        case SBG_ERR_CUDA: return "CUDA error";
        case SBG_ERR_NO_MEMORY: return "out of device memory";
        case SBG_ERR_UNSUPPORTED: return "unsupported size";
        case SBG_ERR_CAPTURING: return "workspace growth during stream capture";
        case SBG_ERR_INTERNAL: return "internal error";
        default: return "unknown status";
    }
}

const char* sbg_last_error(void) { return g_last_error.c_str(); }

void sbg_solver_options_init(sbg_solver_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tuning_mode = SBG_TUNING_SUGGESTED;
    o->cache_mode = SBG_CACHE_AUTO;
    o->precision = SBG_PRECISION_FP64;
}

int sbg_solver_create(int n, int device_id, const sbg_solver_options* opts, sbg_solver** out) {
    return guarded([&] { create_solver(n, device_id, opts, out); });
}

int sbg_solver_destroy(sbg_solver* s) {
    return guarded([&] { delete s; });
}

int sbg_solver_launch(sbg_solver* s, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B, double* d_W,
                      cuDoubleComplex* d_X, int* d_info, int batch, cudaStream_t stream) {
    return guarded([&] {
        if (!s) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        DeviceGuard g(s->device);
        s->launch(c2(d_A), c2(d_B), d_W, c2(d_X), d_info, batch, stream);
    });
}

int sbg_solver_launch_chunked(sbg_solver* s, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B,
                              double* d_W, cuDoubleComplex* d_X, int* d_info, int total, int chunk_size,
                              int num_streams, const cudaStream_t* streams) {
    return guarded([&] {
        if (!s) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        if (total < 0) throw Error(SBG_ERR_INVALID_VALUE, "total < 0");
        if (total == 0) return;
        if (chunk_size <= 0) throw Error(SBG_ERR_INVALID_VALUE, "launch_chunked: chunk_size must be > 0");
        if (num_streams <= 0 || !streams)
            throw Error(SBG_ERR_INVALID_VALUE, "launch_chunked: need num_streams > 0 streams");
        DeviceGuard g(s->device);
        const size_t nn = static_cast<size_t>(s->n) * s->n;
        int idx = 0;
        for (int off = 0; off < total; off += chunk_size, ++idx) {
            const int cnt = std::min(chunk_size, total - off);
            const int k = idx % num_streams;        // one workspace per stream: chunks in flight never share
            s->launch(c2(d_A) + nn * off, c2(d_B) + nn * off, d_W + static_cast<size_t>(s->n) * off,
                      c2(d_X) + nn * off, d_info + off, cnt, streams[k]);
        }
    });
}

int sbg_solver_solve_host(sbg_solver* s, const cuDoubleComplex* h_A, const cuDoubleComplex* h_B, double* h_W,
                          cuDoubleComplex* h_X, int* h_info, int batch, int chunk_size, int num_streams) {
    return guarded([&] {
        if (!s) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        DeviceGuard g(s->device);
        s->solve_host(c2(h_A), c2(h_B), h_W, c2(h_X), h_info, batch, chunk_size, num_streams);
    });
}

int sbg_solver_host_transfer_bytes(const sbg_solver* s, long long* h2d_bytes, long long* d2h_bytes) {
    return guarded([&] {
        if (!s) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        if (h2d_bytes) *h2d_bytes = s->last_h2d_bytes;
        if (d2h_bytes) *d2h_bytes = s->last_d2h_bytes;
    });
}

int sbg_solver_refine_redo_pairs(sbg_solver* s, long long* count, int reset) {
    return guarded([&] {
        if (!s || !count) throw Error(SBG_ERR_INVALID_VALUE, "null argument");
        *count = 0;
        if (!s->d_redo) return;                 // FP64 solver, or no launch yet
        DeviceGuard g(s->device);
        unsigned long long v = 0;
        check_cuda(cudaMemcpy(&v, s->d_redo, sizeof(v), cudaMemcpyDeviceToHost), "D2H redo counter");
        *count = static_cast<long long>(v);
        if (reset) check_cuda(cudaMemset(s->d_redo, 0, sizeof(v)), "cudaMemset(redo counter)");
    });
}

int sbg_solver_enable_stage_timing(sbg_solver* s, int enable) {
    return guarded([&] {
        if (!s) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        s->timing = enable != 0;
    });
}

int sbg_solver_read_stage_times(sbg_solver* s, double* ms, int* launches) {
    return guarded([&] {
        if (!s || !ms || !launches) throw Error(SBG_ERR_INVALID_VALUE, "null argument");
        DeviceGuard g(s->device);
        std::vector<sbg_solver::StageEvents> evs;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            evs.swap(s->stage_events);
        }
        for (int k = 0; k < 4; ++k) { ms[k] = 0.0; launches[k] = 0; }
        for (auto& e : evs) {
            check_cuda(cudaEventSynchronize(e.b), "cudaEventSynchronize");
            float t = 0.f;
            check_cuda(cudaEventElapsedTime(&t, e.a, e.b), "cudaEventElapsedTime");
            ms[e.stage] += t;
            launches[e.stage] += e.kernels;
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
    });
}

int sbg_solver_reserve(sbg_solver* s, int pairs, int stream_slots) {
    return guarded([&] {
        if (!s || pairs < 0 || stream_slots < 1) throw Error(SBG_ERR_INVALID_VALUE, "bad reserve arguments");
        DeviceGuard g(s->device);
        const int cap = std::min(std::max(pairs, 1), s->chunk_pairs);
        for (int i = 0; i < stream_slots; ++i) s->workspace(i, cap, nullptr);
    });
}

size_t sbg_workspace_bytes_per_pair(int n, int precision) {
    return n > 0 ? sbg::workspace_bytes_per_pair(n, precision == SBG_PRECISION_MIXED) : 0;
}

int sbg_selftest_reciprocal(const double* d_u, double* d_r, int count, cudaStream_t stream) {
    return guarded([&] {
        if (count < 0) throw Error(SBG_ERR_INVALID_VALUE, "count < 0");
        if (count > 0 && (!d_u || !d_r)) throw Error(SBG_ERR_INVALID_VALUE, "null device pointer");
        check_cuda(sbg::launch_selftest_recip(d_u, d_r, count, stream), "reciprocal self-test kernel");
    });
}

int sbg_selftest_fp64_fma(double* d_out, int blocks, int iters, cudaStream_t stream) {
    return guarded([&] {
        if (!d_out || blocks <= 0 || iters <= 0) throw Error(SBG_ERR_INVALID_VALUE, "bad FMA probe arguments");
        check_cuda(sbg::launch_selftest_fp64_fma(d_out, blocks, iters, stream), "FP64 FMA probe kernel");
    });
}

size_t sbg_workspace_bytes(int n, int precision, int pairs) {
    return n > 0 && pairs > 0 ? sbg::workspace_bytes(n, pairs, precision == SBG_PRECISION_MIXED) : 0;
}

int sbg_solver_matrix_size(const sbg_solver* s) { return s ? s->n : 0; }
int sbg_solver_schedule(const sbg_solver* s, int* out8) {
    return guarded([&] {
        if (!s || !out8) throw Error(SBG_ERR_INVALID_VALUE, "null argument");
        const sbg::Schedule& c = s->sched;
        const int v[8] = {c.hetrd_threads, c.pair_warps, c.col_exact, c.back_lanes, c.ql_warps, c.chain_threads,
                          c.back_qpass, c.reduce_tc};
        for (int i = 0; i < 8; ++i) out8[i] = v[i];
    });
}

int sbg_solver_set_schedule(sbg_solver* s, const int* in8) {
    return guarded([&] {
        if (!s || !in8) throw Error(SBG_ERR_INVALID_VALUE, "null argument");
        sbg::Schedule c;
        c.hetrd_threads = in8[0];
        c.pair_warps = in8[1];
        c.col_exact = in8[2];
        c.back_lanes = in8[3];
        c.ql_warps = in8[4];
        c.chain_threads = in8[5];
        c.back_qpass = in8[6];
        c.reduce_tc = in8[7];
        const bool ok = (c.hetrd_threads == 128 || c.hetrd_threads == 256) &&
                        (c.reduce_tc == 0 || c.reduce_tc == 1) &&
                        (c.pair_warps == 1 || c.pair_warps == 2 || c.pair_warps == 4) &&
                        (c.col_exact == 0 || c.col_exact == 1) && (c.back_lanes == 1 || c.back_lanes == 2) &&
                        (c.back_qpass == 1 || c.back_qpass == 2) &&
                        c.ql_warps >= 1 && c.ql_warps <= 16 &&
                        (c.chain_threads == 32 || c.chain_threads == 64 || c.chain_threads == 128 ||
                         c.chain_threads == 256);
        if (!ok) throw Error(SBG_ERR_INVALID_VALUE, "schedule value out of range");
        DeviceGuard g(s->device);
        if (!sbg::schedule_fits(s->n, s->precision, c))
            throw Error(SBG_ERR_INVALID_VALUE, "schedule exceeds the device's shared memory for this n");
        std::lock_guard<std::mutex> lock(s->mu);
        s->sched = c;
    });
}

int sbg_solver_batches_per_block(const sbg_solver* s) {
    return s ? (s->n <= 65 ? s->sched.pair_warps : s->sched.ql_warps) : 0;
}
int sbg_solver_block_dim_x(const sbg_solver* s) { return s ? s->sched.hetrd_threads : 0; }
unsigned int sbg_solver_shared_mem_bytes(const sbg_solver* s) {
    if (!s) return 0;
    size_t m = s->n > sbg::kSmallMaxN
                   ? sbg::big_stage_smem_bytes(s->n, s->sched.reduce_tc != 0, s->sched.chain_threads)
                   : std::max(sbg::reduce_smem_bytes(sbg::kReduceFull, s->n), sbg::back_smem_bytes(s->n));
    if (sbg::mixed_big(s->n, s->precision == SBG_PRECISION_MIXED))
        m = std::max(m, std::max(sbg::hetrd_c64_big_smem_bytes(s->n), sbg::refine_big_smem_bytes()));
    return static_cast<unsigned>(m);
}
int sbg_solver_was_autotuned(const sbg_solver* s) { return s ? s->autotuned : 0; }
int sbg_solver_autotune_sweep_ran(const sbg_solver* s) { return s ? s->sweep_ran : 0; }
const char* sbg_solver_cache_layer_used(const sbg_solver* s) { return s ? s->layer : ""; }
int sbg_solver_precision(const sbg_solver* s) { return s ? s->precision : -1; }

int sbg_tuning_table_path(int device_id, char* buf, size_t buflen) {
    return guarded([&] {
        if (!buf || buflen == 0) throw Error(SBG_ERR_INVALID_VALUE, "buffer");
        const std::string p = sbg::tuning_table_path(device_id);
        if (p.size() + 1 > buflen) throw Error(SBG_ERR_INVALID_VALUE, "buffer too small");
        std::memcpy(buf, p.c_str(), p.size() + 1);
    });
}

int sbg_tuning_forget_in_process(void) {
    return guarded([&] { sbg::forget_in_process(); });
}

int sbg_max_n(int precision) {
    int r = 0;
    guarded([&] { r = supported_max_n(precision); });
    return r;
}

// ------------------------------------------------------------------ fixed n = 54 drop-in

void geneig_full_n54_batched_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S, double* d_W,
                                    cuDoubleComplex* d_U, int* d_info, int batch_size, cudaStream_t stream) {
    report_void(guarded([&] {
        if (batch_size <= 0) return;
        default_n54_solver()->launch(c2(d_H), c2(d_S), d_W, c2(d_U), d_info, batch_size, stream);
    }));
}
unsigned int geneig_full_n54_batched_block_dim_x(void) { return sbg::default_schedule(54, SBG_PRECISION_FP64).hetrd_threads; }
unsigned int geneig_full_n54_batched_shared_mem_bytes(void) {
    return static_cast<unsigned>(std::max(sbg::reduce_smem_bytes(sbg::kReduceFull, 54), sbg::back_smem_bytes(54)));
}

void chol_n54_launch(const cuDoubleComplex* d_S, cuDoubleComplex* d_L, int* d_info, cudaStream_t stream) {
    report_void(guarded([&] {
        sbg::Workspace none;
        check_cuda(sbg::launch_reduce(sbg::kReduceChol, nullptr, c2(d_S), 54, 1, none, c2(d_L), d_info,
                                      sbg::default_schedule(54, SBG_PRECISION_FP64).shape(), stream),
                   "chol kernel");
    }));
}
unsigned int chol_n54_block_dim_x(void) { return sbg::default_schedule(54, SBG_PRECISION_FP64).hetrd_threads; }
unsigned int chol_n54_shared_mem_bytes(void) { return static_cast<unsigned>(sbg::reduce_smem_bytes(sbg::kReduceChol, 54)); }

void geneig_reduce_n54_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S, cuDoubleComplex* d_M,
                              int* d_info, cudaStream_t stream) {
    report_void(guarded([&] {
        sbg::Workspace none;
        check_cuda(sbg::launch_reduce(sbg::kReduceHegst, c2(d_H), c2(d_S), 54, 1, none, c2(d_M), d_info,
                                      sbg::default_schedule(54, SBG_PRECISION_FP64).shape(), stream),
                   "reduce kernel");
    }));
}
unsigned int geneig_reduce_n54_block_dim_x(void) { return sbg::default_schedule(54, SBG_PRECISION_FP64).hetrd_threads; }
unsigned int geneig_reduce_n54_shared_mem_bytes(void) { return static_cast<unsigned>(sbg::reduce_smem_bytes(sbg::kReduceHegst, 54)); }

void geneig_reduce_eig_n54_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S, double* d_W,
                                  cuDoubleComplex* d_V, int* d_info, cudaStream_t stream) {
    report_void(guarded([&] {
        sbg_solver* s = default_n54_solver();
        sbg::Workspace ws = s->workspace(0, 1, stream);
        check_cuda(sbg::launch_reduce(sbg::kReduceFull, c2(d_H), c2(d_S), 54, 1, ws, c2(d_V), d_info,
                                      s->sched.shape(), stream), "reduce kernel");
        check_cuda(sbg::launch_hetrd(54, 1, c2(d_V), ws, d_info, s->sched.shape(), stream), "hetrd kernel");
        check_cuda(sbg::launch_ql_logged(54, 1, ws, d_W, c2(d_V), d_info, false, s->sched.chain_threads,
                                         s->sched.ql_warps, stream), "QL kernels");
        check_cuda(sbg::launch_back(sbg::kBackQOnly, 54, 1, ws, c2(d_V), d_info, s->sched.shape(), stream),
                   "back kernel");
    }));
}
unsigned int geneig_reduce_eig_n54_block_dim_x(void) { return sbg::default_schedule(54, SBG_PRECISION_FP64).hetrd_threads; }
unsigned int geneig_reduce_eig_n54_shared_mem_bytes(void) { return geneig_full_n54_batched_shared_mem_bytes(); }
unsigned int geneig_reduce_eig_n54_chol_smem_bytes(void) { return static_cast<unsigned>(sbg::reduce_smem_bytes(sbg::kReduceFull, 54)); }
unsigned int geneig_reduce_eig_n54_heev_smem_bytes(void) {
    return static_cast<unsigned>(sbg::ql_apply_smem_bytes(54, sbg::default_schedule(54, SBG_PRECISION_FP64).ql_warps, false));
}
unsigned int geneig_reduce_eig_n54_heev_workspace(void) {
    return static_cast<unsigned>(sbg::workspace_bytes_per_pair(54) / 16);
}

void geneig_full_n54_launch(const cuDoubleComplex* d_H, const cuDoubleComplex* d_S, double* d_W,
                            cuDoubleComplex* d_U, int* d_info, cudaStream_t stream) {
    geneig_full_n54_batched_launch(d_H, d_S, d_W, d_U, d_info, 1, stream);
}
unsigned int geneig_full_n54_block_dim_x(void) { return geneig_full_n54_batched_block_dim_x(); }
unsigned int geneig_full_n54_shared_mem_bytes(void) { return geneig_full_n54_batched_shared_mem_bytes(); }

void geneig_finish_n54_launch(const cuDoubleComplex* d_L, const cuDoubleComplex* d_M, double* d_W,
                              cuDoubleComplex* d_U, int* d_info, int batch_size, cudaStream_t stream) {
    report_void(guarded([&] {
        if (batch_size <= 0) return;
        sbg_solver* s = default_n54_solver();
        const size_t nn = 54 * 54;
        const int cap = std::min(batch_size, s->chunk_pairs);
        sbg::Workspace ws = s->workspace(0, cap, stream);
        for (int off = 0; off < batch_size; off += ws.capacity) {
            const int cnt = std::min(ws.capacity, batch_size - off);
            check_cuda(sbg::launch_reduce(sbg::kReduceFromLM, nullptr, c2(d_L) + nn * off, 54, cnt, ws,
                                          nullptr, d_info + off, s->sched.shape(), stream), "reduce kernel");
            check_cuda(sbg::launch_hetrd(54, cnt, c2(d_M) + nn * off, ws, d_info + off, s->sched.shape(), stream),
                       "hetrd kernel");
            check_cuda(sbg::launch_ql_logged(54, cnt, ws, d_W + 54 * off, c2(d_U) + nn * off, d_info + off, false,
                                             s->sched.chain_threads, s->sched.ql_warps, stream), "QL kernels");
            check_cuda(sbg::launch_back(sbg::kBackFull, 54, cnt, ws, c2(d_U) + nn * off, d_info + off,
                                        s->sched.shape(), stream), "back kernel");
        }
    }));
}
unsigned int geneig_finish_n54_block_dim_x(void) { return geneig_full_n54_batched_block_dim_x(); }
unsigned int geneig_finish_n54_shared_mem_bytes(void) { return geneig_full_n54_batched_shared_mem_bytes(); }

}  // extern "C"
