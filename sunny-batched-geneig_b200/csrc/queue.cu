// Uneven-n batches in one launch call (sbg_queue_* / sbg_launch_queue).
//
// The reference has no such path: its runtime-n solver (src/nvrtc/nvrtc_solver.hpp:99-145)
// serves one n per instance, so a mixed batch needs one solver and one launch per n.
// Here a queue is planned once for the sequence of orders n[0..count): the pairs are
// bucketed by n (largest n first, so the longest buckets start earliest), every bucket
// gets its own solver (with the per-n schedule from the tuning table or the autotuner),
// staging buffers for one chunk of its pairs and a stream.  A launch replays a CUDA
// graph that forks one branch per bucket off the caller's stream; a branch loops over
// its chunks: gather the chunk's pairs out of the packed inputs, run the stage kernels
// of that n, scatter X, W and info back.  The branches run concurrently, so a bucket
// that cannot fill the GPU on its own overlaps with the others.  The graph is captured
// on the first launch and re-captured (then updated in place) only when the caller's
// buffers change.
//
// Packed layout: pair p's A, B and X start at element mat_off[p] = sum_{q<p} n[q]^2
// (column-major, lda = n[p]), its W at vec_off[p] = sum_{q<p} n[q], its info at p.
#include "solver.h"

#include <cstdio>
#include <functional>
#include <map>
#include <memory>

namespace {

constexpr int kCopyThreads = 256;

// Pair idx[first + i] of the packed A, B -> slot i of the bucket's staging buffers.
__global__ void __launch_bounds__(kCopyThreads) k_gather(const double2* __restrict__ A,
                                                         const double2* __restrict__ B,
                                                         const long long* __restrict__ mat_off,
                                                         const int* __restrict__ idx, int first, int count, int nn,
                                                         double2* __restrict__ As, double2* __restrict__ Bs) {
    const int i = blockIdx.x;
    if (i >= count) return;
    const long long o = mat_off[idx[first + i]];
    const double2* a = A + o;
    const double2* b = B + o;
    double2* as = As + static_cast<size_t>(i) * nn;
    double2* bs = Bs + static_cast<size_t>(i) * nn;
    for (int t = threadIdx.x; t < nn; t += kCopyThreads) { as[t] = a[t]; bs[t] = b[t]; }
}

// Slot i of the bucket's X, W, info staging -> pair idx[first + i] of the packed outputs.
__global__ void __launch_bounds__(kCopyThreads) k_scatter(const double2* __restrict__ Xs,
                                                          const double* __restrict__ Ws,
                                                          const int* __restrict__ Is,
                                                          const long long* __restrict__ mat_off,
                                                          const long long* __restrict__ vec_off,
                                                          const int* __restrict__ idx, int first, int count, int n,
                                                          double2* __restrict__ X, double* __restrict__ W,
                                                          int* __restrict__ info) {
    const int i = blockIdx.x;
    if (i >= count) return;
    const int p = idx[first + i];
    const int nn = n * n;
    double2* x = X + mat_off[p];
    const double2* xs = Xs + static_cast<size_t>(i) * nn;
    for (int t = threadIdx.x; t < nn; t += kCopyThreads) x[t] = xs[t];
    double* w = W + vec_off[p];
    for (int t = threadIdx.x; t < n; t += kCopyThreads) w[t] = Ws[static_cast<size_t>(i) * n + t];
    if (threadIdx.x == 0) info[p] = Is[i];
}

struct Bucket {
    int n = 0;
    int count = 0;
    int chunk = 0;
    int precision = SBG_PRECISION_FP64;
    std::vector<int> pairs;
    int* d_idx = nullptr;
    sbg_solver* solver = nullptr;
    double2* As = nullptr;
    double2* Bs = nullptr;
    double2* Xs = nullptr;
    double* Ws = nullptr;
    int* Is = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
};

// Device bytes one pair of order n takes in a bucket: staging plus solver workspace.
size_t bucket_bytes_per_pair(int n, bool mixed) {
    const size_t nn = static_cast<size_t>(n) * n;
    return 48 * nn + 8 * static_cast<size_t>(n) + 4 + sbg::workspace_bytes_per_pair(n, mixed);
}

}  // namespace

struct sbg_queue {
    int device = 0;
    int count = 0;
    long long mat_total = 0;
    long long vec_total = 0;
    long long* d_mat_off = nullptr;
    long long* d_vec_off = nullptr;
    std::vector<Bucket> buckets;
    cudaStream_t capture_stream = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int graph_builds = 0;
    std::mutex mu;

    ~sbg_queue() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& b : buckets) {
            if (b.solver) sbg_solver_destroy(b.solver);
            for (void* p : {static_cast<void*>(b.d_idx), static_cast<void*>(b.As), static_cast<void*>(b.Bs),
                            static_cast<void*>(b.Xs), static_cast<void*>(b.Ws), static_cast<void*>(b.Is)})
                if (p) cudaFree(p);
            if (b.stream) cudaStreamDestroy(b.stream);
            if (b.done) cudaEventDestroy(b.done);
        }
        if (d_mat_off) cudaFree(d_mat_off);
        if (d_vec_off) cudaFree(d_vec_off);
        if (fork) cudaEventDestroy(fork);
        if (capture_stream) cudaStreamDestroy(capture_stream);
        cudaSetDevice(prev);
    }

    // Enqueues the whole queue on s0 (the capture stream).
    void enqueue(cudaStream_t s0, const double2* A, const double2* B, double* W, double2* X, int* info) {
        check_cuda(cudaEventRecord(fork, s0), "cudaEventRecord");
        for (auto& b : buckets) {
            check_cuda(cudaStreamWaitEvent(b.stream, fork, 0), "cudaStreamWaitEvent");
            const int nn = b.n * b.n;
            for (int first = 0; first < b.count; first += b.chunk) {
                const int cnt = std::min(b.chunk, b.count - first);
                k_gather<<<cnt, kCopyThreads, 0, b.stream>>>(A, B, d_mat_off, b.d_idx, first, cnt, nn, b.As, b.Bs);
                check_cuda(cudaGetLastError(), "gather kernel");
                b.solver->launch(b.As, b.Bs, b.Ws, b.Xs, b.Is, cnt, b.stream);
                k_scatter<<<cnt, kCopyThreads, 0, b.stream>>>(b.Xs, b.Ws, b.Is, d_mat_off, d_vec_off, b.d_idx, first,
                                                              cnt, b.n, X, W, info);
                check_cuda(cudaGetLastError(), "scatter kernel");
            }
            check_cuda(cudaEventRecord(b.done, b.stream), "cudaEventRecord");
            check_cuda(cudaStreamWaitEvent(s0, b.done, 0), "cudaStreamWaitEvent");
        }
    }

    void launch(const double2* A, const double2* B, double* W, double2* X, int* info, cudaStream_t stream) {
        if (count == 0) return;
        if (!A || !B || !W || !X || !info) throw Error(SBG_ERR_INVALID_VALUE, "null device pointer");
        std::lock_guard<std::mutex> lock(mu);
        const void* k[5] = {A, B, W, X, info};
        bool same = exec != nullptr;
        for (int i = 0; i < 5; ++i) same = same && key[i] == k[i];
        if (!same) {
            cudaGraph_t g = nullptr;
            // Relaxed: the first capture may be the first use of a stage kernel, whose one-time
            // shared-memory attribute call is not a stream operation.
            check_cuda(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
            try {
                enqueue(capture_stream, A, B, W, X, info);
            } catch (...) {
                cudaStreamEndCapture(capture_stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            check_cuda(cudaStreamEndCapture(capture_stream, &g), "cudaStreamEndCapture");
            bool updated = false;
            if (exec) {
                cudaGraphExecUpdateResultInfo res;
                updated = cudaGraphExecUpdate(exec, g, &res) == cudaSuccess;
                if (!updated) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(exec);
                    exec = nullptr;
                }
            }
            if (!updated) check_cuda(cudaGraphInstantiate(&exec, g, 0), "cudaGraphInstantiate");
            if (graph) cudaGraphDestroy(graph);
            graph = g;
            for (int i = 0; i < 5; ++i) key[i] = k[i];
            ++graph_builds;
        }
        check_cuda(cudaGraphLaunch(exec, stream), "cudaGraphLaunch");
    }
};

namespace {

void create_queue(const int* n_host, int count, int device, const sbg_solver_options* o, sbg_queue** out) {
    if (!out) throw Error(SBG_ERR_INVALID_VALUE, "out == NULL");
    *out = nullptr;
    if (count < 0) throw Error(SBG_ERR_INVALID_VALUE, "count < 0");
    if (count > 0 && !n_host) throw Error(SBG_ERR_INVALID_VALUE, "n == NULL");
    sbg_solver_options opts;
    sbg_solver_options_init(&opts);
    if (o) opts = *o;
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) throw Error(SBG_ERR_INVALID_VALUE, "device_id out of range");
    DeviceGuard g(device);
    const int max_fp64 = sbg_max_n(SBG_PRECISION_FP64);
    const int max_mixed = sbg_max_n(SBG_PRECISION_MIXED);
    std::unique_ptr<sbg_queue> q(new sbg_queue);
    q->device = device;
    q->count = count;
    std::vector<long long> mat_off(count), vec_off(count);
    std::map<int, std::vector<int>, std::greater<int>> by_n;
    long long mo = 0, vo = 0;
    for (int p = 0; p < count; ++p) {
        const int n = n_host[p];
        if (n < 1 || n > max_fp64)
            throw Error(n < 1 ? SBG_ERR_INVALID_VALUE : SBG_ERR_UNSUPPORTED,
                        "pair " + std::to_string(p) + ": n = " + std::to_string(n) + " outside 1.." +
                            std::to_string(max_fp64));
        mat_off[p] = mo;
        vec_off[p] = vo;
        mo += static_cast<long long>(n) * n;
        vo += n;
        by_n[n].push_back(p);
    }
    q->mat_total = mo;
    q->vec_total = vo;
    if (count == 0) { *out = q.release(); return; }
    check_cuda(cudaMalloc(&q->d_mat_off, sizeof(long long) * count), "cudaMalloc(queue offsets)");
    check_cuda(cudaMalloc(&q->d_vec_off, sizeof(long long) * count), "cudaMalloc(queue offsets)");
    check_cuda(cudaMemcpy(q->d_mat_off, mat_off.data(), sizeof(long long) * count, cudaMemcpyHostToDevice), "H2D");
    check_cuda(cudaMemcpy(q->d_vec_off, vec_off.data(), sizeof(long long) * count, cudaMemcpyHostToDevice), "H2D");
    check_cuda(cudaStreamCreateWithFlags(&q->capture_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreateWithFlags(&q->fork, cudaEventDisableTiming), "cudaEventCreate");
    // Staging + workspace per bucket: half of the free device memory shared by the buckets, between
    // 1 and 8 GiB.  Bigger chunks mean fewer, fuller launches per bucket: with 1 GiB the n = 128
    // bucket of the 500,000-pair uneven batch ran ~36 chunks of ~700 pairs (2.4 waves of its
    // one-CTA-per-pair kernels) back to back.
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t budget = std::min<size_t>(size_t(8) << 30,
                                           std::max<size_t>(size_t(1) << 30, free_b / 2 / by_n.size()));
    for (auto& kv : by_n) {
        q->buckets.emplace_back();
        Bucket& b = q->buckets.back();
        b.n = kv.first;
        b.pairs = std::move(kv.second);
        b.count = static_cast<int>(b.pairs.size());
        b.precision = (opts.precision == SBG_PRECISION_MIXED && b.n <= max_mixed) ? SBG_PRECISION_MIXED
                                                                                  : SBG_PRECISION_FP64;
        const size_t per = bucket_bytes_per_pair(b.n, b.precision == SBG_PRECISION_MIXED);
        int chunk = static_cast<int>(std::max<size_t>(256, budget / per));
        if (opts.workspace_pairs > 0) chunk = opts.workspace_pairs;
        b.chunk = std::min(chunk, b.count);
        sbg_solver_options so = opts;
        so.precision = b.precision;
        so.workspace_pairs = b.chunk;
        create_solver(b.n, device, &so, &b.solver);
        if (int st = sbg_solver_reserve(b.solver, b.chunk, 1))
            throw Error(st, std::string("queue workspace: ") + sbg_last_error());
        const size_t nn = static_cast<size_t>(b.n) * b.n, c = static_cast<size_t>(b.chunk);
        check_cuda(cudaMalloc(&b.d_idx, sizeof(int) * b.count), "cudaMalloc(queue index)");
        check_cuda(cudaMemcpy(b.d_idx, b.pairs.data(), sizeof(int) * b.count, cudaMemcpyHostToDevice), "H2D");
        check_cuda(cudaMalloc(&b.As, 16 * nn * c), "cudaMalloc(queue staging)");
        check_cuda(cudaMalloc(&b.Bs, 16 * nn * c), "cudaMalloc(queue staging)");
        check_cuda(cudaMalloc(&b.Xs, 16 * nn * c), "cudaMalloc(queue staging)");
        check_cuda(cudaMalloc(&b.Ws, 8 * static_cast<size_t>(b.n) * c), "cudaMalloc(queue staging)");
        check_cuda(cudaMalloc(&b.Is, 4 * c), "cudaMalloc(queue staging)");
        check_cuda(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming), "cudaEventCreate");
    }
    *out = q.release();
}

}  // namespace

extern "C" {

int sbg_queue_create(const int* n, int count, int device_id, const sbg_solver_options* opts, sbg_queue** out) {
    return guarded([&] { create_queue(n, count, device_id, opts, out); });
}

int sbg_queue_destroy(sbg_queue* q) {
    return guarded([&] { delete q; });
}

int sbg_launch_queue(sbg_queue* q, const cuDoubleComplex* d_A, const cuDoubleComplex* d_B, double* d_W,
                     cuDoubleComplex* d_X, int* d_info, cudaStream_t stream) {
    return guarded([&] {
        if (!q) throw Error(SBG_ERR_INVALID_VALUE, "queue == NULL");
        DeviceGuard g(q->device);
        q->launch(reinterpret_cast<const double2*>(d_A), reinterpret_cast<const double2*>(d_B), d_W,
                  reinterpret_cast<double2*>(d_X), d_info, stream);
    });
}

int sbg_queue_size(const sbg_queue* q) { return q ? q->count : 0; }
long long sbg_queue_matrix_elements(const sbg_queue* q) { return q ? q->mat_total : 0; }
long long sbg_queue_vector_elements(const sbg_queue* q) { return q ? q->vec_total : 0; }
int sbg_queue_buckets(const sbg_queue* q) { return q ? static_cast<int>(q->buckets.size()) : 0; }
int sbg_queue_graph_builds(const sbg_queue* q) { return q ? q->graph_builds : 0; }

int sbg_queue_bucket(const sbg_queue* q, int i, int* n, int* count, int* chunk, int* precision, int* was_autotuned) {
    return guarded([&] {
        if (!q || i < 0 || i >= static_cast<int>(q->buckets.size())) throw Error(SBG_ERR_INVALID_VALUE, "bad bucket");
        const Bucket& b = q->buckets[i];
        if (n) *n = b.n;
        if (count) *count = b.count;
        if (chunk) *chunk = b.chunk;
        if (precision) *precision = b.precision;
        if (was_autotuned) *was_autotuned = sbg_solver_was_autotuned(b.solver);
    });
}

}  // extern "C"
