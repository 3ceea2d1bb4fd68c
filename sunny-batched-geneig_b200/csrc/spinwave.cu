// Spin-wave q-sweeps on the GPU: the step ahead of the solve (assembling the pairs of
// every q from one cell's bond table) and the step after it (contracting each
// eigenvector to an intensity), both with no counterpart in the reference.  The
// reference's intended caller (Sunny.jl) assembles A(q), B(q) on the host and ships
// 2 x 16 n^2 bytes per q to the solver, then reads 16 n^2 bytes of eigenvectors back
// per q; with the model on the GPU a sweep moves 24 bytes of q in and W plus n
// intensities out per q.
//
// Model of one cell: N sites (n = 2N), bonds k = (i, j, a, b, c, d) with complex a, b,
// real c and displacement d; per q:
//   P(q)_ij += a/2 e^{i q.d},  P(q)_ji += conj(a/2 e^{i q.d}),
//   Q(q)_ij += b/2 e^{i q.d},  Q(q)_ji += b/2 e^{i q.d},
//   P_ii -= c/2,  P_jj -= c/2,
// and A = diag(I_N, -I_N), B(q) = [[P, Q], [conj Q, conj P]] + field I.
// Intensity of eigenpair m of pair q (x_m B-orthonormal, lambda_m from W):
//   I_m(q) = |sum_{i<N} e^{-i q.r_i} (x_m[i] + x_m[N+i])|^2 / (N |lambda_m|).
//
// Layout in HBM: the bond table is preprocessed on the host into, per N x N block,
// a dense map from entry (r, c) to a list of bond contributions in bond order (P:
// bond index << 1 | conjugate flag; Q: bond index, a bond with i = j listed twice),
// so each entry of B is a fixed-order sum (deterministic, no atomics).  q is
// double[nq][3]; A, B, X, W and info use the solver's layout.
#include "common.cuh"
#include "solver.h"

#include <cmath>
#include <cstring>
#include <memory>

namespace {

constexpr int kAssembleThreads = 256;
constexpr int kIntensityThreads = 128;

// Device copy of a cell, one allocation: doubles first, then ints.
struct SwTables {
    int N = 0, nb = 0;
    double field = 0.0;
    const double2* half_a = nullptr;    // a/2 per bond
    const double2* half_b = nullptr;    // b/2 per bond
    const double* disp = nullptr;       // d per bond, [nb][3]
    const double* onsite = nullptr;     // sum of -c/2 per site, [N]
    const double* pos = nullptr;        // r per site, [N][3] (zeros when none given)
    const int* mapP = nullptr;          // [N*N] entry r + N c -> list index, or -1
    const int* ptrP = nullptr;
    const int* listP = nullptr;
    const int* mapQ = nullptr;
    const int* ptrQ = nullptr;
    const int* listQ = nullptr;
    const int* entP = nullptr;          // list index k -> its entry r + N c (P, then Q)
    const int* entQ = nullptr;
    int nP = 0, nQ = 0;                 // entries with contributions
};

// Sum of the contributions t[list[ptr[k] ..]] (conjugated where flagged) of list entry k.
__device__ __forceinline__ double2 list_sum(const int* ptr, const int* list, int k, const double2* t, bool flagged) {
    double2 v = make_double2(0.0, 0.0);
    for (int j = ptr[k]; j < ptr[k + 1]; ++j) {
        const int e = list[j];
        double2 c = t[flagged ? (e >> 1) : e];
        if (flagged && (e & 1)) c.y = -c.y;
        v.x += c.x;
        v.y += c.y;
    }
    return v;
}

// One CTA per q: the bond phases into shared memory; B(q) (and, when A != nullptr, the metric A)
// zero-filled with plain coalesced stores, then only the entries with bond contributions and the
// diagonal written (a third of B at n = 54): each a fixed-order sum, so B is bit-reproducible.
__global__ void __launch_bounds__(kAssembleThreads) k_sw_assemble(SwTables T, const double* __restrict__ qv, int nq,
                                                                   double2* __restrict__ A, double2* __restrict__ B) {
    const int p = blockIdx.x;
    if (p >= nq) return;
    extern __shared__ __align__(16) double2 sw_smem[];
    double2* ta = sw_smem;              // a/2 e^{i q.d}
    double2* tb = sw_smem + T.nb;       // b/2 e^{i q.d}
    const double q0 = qv[3 * p], q1 = qv[3 * p + 1], q2 = qv[3 * p + 2];
    for (int k = threadIdx.x; k < T.nb; k += kAssembleThreads) {
        const double* d = T.disp + 3 * k;
        double s, c;
        sincos(q0 * d[0] + q1 * d[1] + q2 * d[2], &s, &c);
        const double2 ph = make_double2(c, s);
        ta[k] = sbg::cmul(T.half_a[k], ph);
        tb[k] = sbg::cmul(T.half_b[k], ph);
    }
    const int N = T.N, n = 2 * N, nn = n * n;
    double2* Bp = B + static_cast<size_t>(nn) * p;
    double2* Ap = A ? A + static_cast<size_t>(nn) * p : nullptr;
    const double2 zero = make_double2(0.0, 0.0);
    for (int e = threadIdx.x; e < nn; e += kAssembleThreads) {
        Bp[e] = zero;
        if (Ap) Ap[e] = zero;
    }
    __syncthreads();                    // phases ready; zeros ordered before the values below
    const size_t ldn = static_cast<size_t>(n);
    for (int k = threadIdx.x; k < T.nP; k += kAssembleThreads) {      // P off the diagonal: P, conj(P) blocks
        const int idx = T.entP[k], c = idx / N, r = idx - c * N;
        if (r == c) continue;
        const double2 v = list_sum(T.ptrP, T.listP, k, ta, true);
        Bp[r + ldn * c] = v;
        Bp[(N + r) + ldn * (N + c)] = make_double2(v.x, -v.y);
    }
    for (int r = threadIdx.x; r < N; r += kAssembleThreads) {         // the diagonal: bonds, on-site, field
        const int k = T.mapP[r + N * r];
        double2 v = k >= 0 ? list_sum(T.ptrP, T.listP, k, ta, true) : zero;
        v.x += T.onsite[r];
        Bp[r + ldn * r] = make_double2(v.x + T.field, v.y);
        Bp[(N + r) + ldn * (N + r)] = make_double2(v.x + T.field, -v.y);
        if (Ap) {
            Ap[r + ldn * r] = make_double2(1.0, 0.0);
            Ap[(N + r) + ldn * (N + r)] = make_double2(-1.0, 0.0);
        }
    }
    for (int k = threadIdx.x; k < T.nQ; k += kAssembleThreads) {      // Q and conj(Q) blocks
        const int idx = T.entQ[k], c = idx / N, r = idx - c * N;
        const double2 v = list_sum(T.ptrQ, T.listQ, k, tb, false);
        Bp[r + ldn * (N + c)] = v;
        Bp[(N + r) + ldn * c] = make_double2(v.x, -v.y);
    }
}

// The metric A = diag(I_N, -I_N) for `count` pairs (the solve's A never changes).
__global__ void __launch_bounds__(kAssembleThreads) k_sw_metric(int N, long long total, double2* __restrict__ A) {
    const int n = 2 * N;
    const long long nn = static_cast<long long>(n) * n;
    for (long long e = blockIdx.x * static_cast<long long>(kAssembleThreads) + threadIdx.x; e < total;
         e += static_cast<long long>(gridDim.x) * kAssembleThreads) {
        const int l = static_cast<int>(e % nn);
        const int col = l / n, row = l - col * n;
        A[e] = make_double2(row == col ? (row < N ? 1.0 : -1.0) : 0.0, 0.0);
    }
}

// One CTA per q, a warp per eigenvector at a time, lanes over sites (coalesced reads of
// x_m[i] and x_m[N+i]); the site phases e^{-i q.r_i} are computed once per q.
__global__ void __launch_bounds__(kIntensityThreads) k_sw_intensity(SwTables T, const double* __restrict__ qv, int nq,
                                                                     const double* __restrict__ W,
                                                                     const double2* __restrict__ X,
                                                                     const int* __restrict__ info,
                                                                     double* __restrict__ I) {
    const int p = blockIdx.x;
    if (p >= nq) return;
    extern __shared__ __align__(16) double2 sw_smem[];
    const int N = T.N, n = 2 * N;
    const double q0 = qv[3 * p], q1 = qv[3 * p + 1], q2 = qv[3 * p + 2];
    for (int i = threadIdx.x; i < N; i += kIntensityThreads) {
        const double* r = T.pos + 3 * i;
        double s, c;
        sincos(q0 * r[0] + q1 * r[1] + q2 * r[2], &s, &c);
        sw_smem[i] = make_double2(c, -s);
    }
    __syncthreads();
    double* Ip = I + static_cast<size_t>(n) * p;
    if (info[p] != 0) {
        for (int m = threadIdx.x; m < n; m += kIntensityThreads) Ip[m] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* Wp = W + static_cast<size_t>(n) * p;
    for (int m = warp; m < n; m += kIntensityThreads / 32) {
        const double2* x = X + (static_cast<size_t>(p) * n + m) * n;
        double2 acc = make_double2(0.0, 0.0);
        for (int i = lane; i < N; i += 32) {
            const double2 u = x[i], v = x[N + i];
            acc = sbg::cfma(sw_smem[i], make_double2(u.x + v.x, u.y + v.y), acc);
        }
        acc.x = sbg::warp_sum(acc.x);
        acc.y = sbg::warp_sum(acc.y);
        if (lane == 0) Ip[m] = (acc.x * acc.x + acc.y * acc.y) / (N * fabs(Wp[m]));
    }
}

}  // namespace

struct sbg_spinwave {
    int device = 0;
    int N = 0;
    int nb = 0;
    void* d_tables = nullptr;
    SwTables T;
    size_t assemble_smem = 0;
    std::mutex mu;
    // Per-stream scratch: A (the metric, written once), B and X of one chunk.
    struct Slot { cudaStream_t stream = nullptr; double2* A = nullptr; double2* B = nullptr; double2* X = nullptr;
                  int capacity = 0; };
    std::vector<std::unique_ptr<Slot>> slots;          // stable addresses: handed out by reference
    // Staging of the host-buffer path, one per internal stream.
    struct Staging { cudaStream_t stream = nullptr; double* q = nullptr; double* W = nullptr; double* I = nullptr;
                     int* info = nullptr; int capacity = 0; };
    std::vector<Staging> staging;
    std::mutex host_mu;                 // one solve_host at a time: they share the staging buffers

    ~sbg_spinwave() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        for (auto& s : slots)
            for (void* p : {static_cast<void*>(s->A), static_cast<void*>(s->B), static_cast<void*>(s->X)})
                if (p) cudaFree(p);
        for (auto& st : staging) {
            if (st.stream) cudaStreamDestroy(st.stream);
            for (void* p : {static_cast<void*>(st.q), static_cast<void*>(st.W), static_cast<void*>(st.I),
                            static_cast<void*>(st.info)})
                if (p) cudaFree(p);
        }
        if (d_tables) cudaFree(d_tables);
        cudaSetDevice(prev);
    }

    int n() const { return 2 * N; }

    void assemble(const double* q, int nq, double2* A, double2* B, cudaStream_t stream) {
        if (nq <= 0) return;
        k_sw_assemble<<<nq, kAssembleThreads, assemble_smem, stream>>>(T, q, nq, A, B);
        check_cuda(cudaGetLastError(), "spin-wave assembly kernel");
    }

    void intensities(const double* q, int nq, const double* W, const double2* X, const int* info, double* I,
                     cudaStream_t stream) {
        if (nq <= 0) return;
        k_sw_intensity<<<nq, kIntensityThreads, sizeof(double2) * N, stream>>>(T, q, nq, W, X, info, I);
        check_cuda(cudaGetLastError(), "spin-wave intensity kernel");
    }

    Slot& slot(cudaStream_t stream, int pairs, bool need_x) {
        std::lock_guard<std::mutex> lock(mu);
        Slot* s = nullptr;
        for (auto& x : slots) if (x->stream == stream) s = x.get();
        if (!s) { slots.emplace_back(new Slot); s = slots.back().get(); s->stream = stream; }
        if (s->capacity >= pairs && (s->X || !need_x)) return *s;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (stream) check_cuda(cudaStreamIsCapturing(stream, &cs), "cudaStreamIsCapturing");
        if (cs != cudaStreamCaptureStatusNone)
            throw Error(SBG_ERR_CAPTURING, "spin-wave scratch must grow while the stream is capturing; "
                                           "run one sweep of this size on the stream before capture");
        const size_t bytes = sizeof(double2) * static_cast<size_t>(n()) * n() * std::max(pairs, s->capacity);
        if (s->capacity < pairs) {
            for (double2** p : {&s->A, &s->B, &s->X}) if (*p) { cudaFree(*p); *p = nullptr; }
            s->capacity = 0;
            check_cuda(cudaMalloc(&s->A, bytes), "cudaMalloc(spin-wave scratch)");
            check_cuda(cudaMalloc(&s->B, bytes), "cudaMalloc(spin-wave scratch)");
            s->capacity = pairs;
            const long long total = static_cast<long long>(n()) * n() * pairs;
            const int grid = static_cast<int>(std::min<long long>((total + kAssembleThreads - 1) / kAssembleThreads,
                                                                  148 * 16));
            k_sw_metric<<<grid, kAssembleThreads, 0, stream>>>(N, total, s->A);
            check_cuda(cudaGetLastError(), "metric kernel");
        }
        if (need_x && !s->X) check_cuda(cudaMalloc(&s->X, bytes), "cudaMalloc(spin-wave scratch)");
        return *s;
    }

    // Assemble, solve and (optionally) contract one sweep, chunk by chunk, on `stream`.
    void solve(sbg_solver* sv, const double* q, int nq, double* W, double2* X, double* I, int* info,
               cudaStream_t stream) {
        if (!sv) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        if (sv->n != n()) throw Error(SBG_ERR_INVALID_VALUE, "solver order " + std::to_string(sv->n) +
                                                                 " != 2 x sites = " + std::to_string(n()));
        if (sv->device != device) throw Error(SBG_ERR_INVALID_VALUE, "solver and model on different devices");
        if (nq < 0) throw Error(SBG_ERR_INVALID_VALUE, "nq < 0");
        if (nq == 0) return;
        if (!q || !W || !info) throw Error(SBG_ERR_INVALID_VALUE, "null device pointer");
        const int chunk = std::min(nq, sv->chunk_pairs);
        Slot& s = slot(stream, chunk, X == nullptr);
        const size_t nn = static_cast<size_t>(n()) * n();
        for (int off = 0; off < nq; off += chunk) {
            const int cnt = std::min(chunk, nq - off);
            const double* qc = q + 3 * static_cast<size_t>(off);
            double* Wc = W + static_cast<size_t>(n()) * off;
            double2* Xc = X ? X + nn * off : s.X;
            assemble(qc, cnt, nullptr, s.B, stream);
            sv->launch(s.A, s.B, Wc, Xc, info + off, cnt, stream);
            if (I) intensities(qc, cnt, Wc, Xc, info + off, I + static_cast<size_t>(n()) * off, stream);
        }
    }

    void solve_host(sbg_solver* sv, const double* hq, int nq, double* hW, double2* hX, double* hI, int* hinfo,
                    int chunk, int nstreams) {
        if (!sv) throw Error(SBG_ERR_INVALID_VALUE, "solver == NULL");
        if (nq < 0 || chunk < 0 || nstreams <= 0) throw Error(SBG_ERR_INVALID_VALUE, "bad solve_host arguments");
        std::lock_guard<std::mutex> serial(host_mu);
        if (nq == 0) return;
        if (!hq || !hW || !hinfo) throw Error(SBG_ERR_INVALID_VALUE, "null host pointer");
        if (chunk == 0) chunk = sv->chunk_pairs;
        chunk = std::min(chunk, nq);
        const size_t nn = static_cast<size_t>(n()) * n();
        {
            std::lock_guard<std::mutex> lock(mu);
            if (static_cast<int>(staging.size()) < nstreams) staging.resize(nstreams);
            for (int i = 0; i < nstreams; ++i) {
                Staging& st = staging[i];
                if (!st.stream) check_cuda(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking), "cudaStreamCreate");
                if (st.capacity < chunk) {
                    for (void** p : {reinterpret_cast<void**>(&st.q), reinterpret_cast<void**>(&st.W),
                                     reinterpret_cast<void**>(&st.I), reinterpret_cast<void**>(&st.info)})
                        if (*p) { cudaFree(*p); *p = nullptr; }
                    check_cuda(cudaMalloc(&st.q, 24 * static_cast<size_t>(chunk)), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.W, 8 * static_cast<size_t>(n()) * chunk), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.I, 8 * static_cast<size_t>(n()) * chunk), "cudaMalloc(staging)");
                    check_cuda(cudaMalloc(&st.info, 4 * static_cast<size_t>(chunk)), "cudaMalloc(staging)");
                    st.capacity = chunk;
                }
            }
        }
        int idx = 0;
        for (int off = 0; off < nq; off += chunk, ++idx) {
            const int cnt = std::min(chunk, nq - off);
            Staging& st = staging[idx % nstreams];
            check_cuda(cudaMemcpyAsync(st.q, hq + 3 * static_cast<size_t>(off), 24 * static_cast<size_t>(cnt),
                                       cudaMemcpyHostToDevice, st.stream), "H2D q");
            solve(sv, st.q, cnt, st.W, nullptr, hI ? st.I : nullptr, st.info, st.stream);
            if (hX) {
                const Slot& s = slot(st.stream, cnt, true);
                check_cuda(cudaMemcpyAsync(hX + nn * off, s.X, 16 * nn * cnt, cudaMemcpyDeviceToHost, st.stream),
                           "D2H X");
            }
            check_cuda(cudaMemcpyAsync(hW + static_cast<size_t>(n()) * off, st.W, 8 * static_cast<size_t>(n()) * cnt,
                                       cudaMemcpyDeviceToHost, st.stream), "D2H W");
            if (hI)
                check_cuda(cudaMemcpyAsync(hI + static_cast<size_t>(n()) * off, st.I,
                                           8 * static_cast<size_t>(n()) * cnt, cudaMemcpyDeviceToHost, st.stream),
                           "D2H intensities");
            check_cuda(cudaMemcpyAsync(hinfo + off, st.info, 4 * static_cast<size_t>(cnt), cudaMemcpyDeviceToHost,
                                       st.stream), "D2H info");
        }
        for (int i = 0; i < nstreams; ++i) check_cuda(cudaStreamSynchronize(staging[i].stream), "cudaStreamSynchronize");
    }
};

namespace {

// Entry (r, c) -> ordered contributions, for one N x N block.
struct EntryLists {
    std::vector<int> map, ptr, list, ent;
    explicit EntryLists(int N) : map(static_cast<size_t>(N) * N, -1), ptr(1, 0) {}
    std::vector<std::vector<int>> pending;
    void add(int idx, int v) {
        if (map[idx] < 0) { map[idx] = static_cast<int>(pending.size()); pending.emplace_back(); ent.push_back(idx); }
        pending[map[idx]].push_back(v);
    }
    void finish() {
        for (auto& l : pending) {
            list.insert(list.end(), l.begin(), l.end());
            ptr.push_back(static_cast<int>(list.size()));
        }
        pending.clear();
    }
};

// k_sw_assemble's dynamic shared-memory limit, raised per device to the largest bond table a
// model on that device needs.
sbg::SmemOptIn g_assemble_attr;

void create_spinwave(int N, int nb, const int* sites, const double* coef, const double* disp, const double* pos,
                     double field, int device, sbg_spinwave** out) {
    if (!out) throw Error(SBG_ERR_INVALID_VALUE, "out == NULL");
    *out = nullptr;
    if (N < 1) throw Error(SBG_ERR_INVALID_VALUE, "n_sites < 1");
    if (nb < 0) throw Error(SBG_ERR_INVALID_VALUE, "n_bonds < 0");
    if (nb > 0 && (!sites || !coef || !disp)) throw Error(SBG_ERR_INVALID_VALUE, "null bond table");
    if (!std::isfinite(field)) throw Error(SBG_ERR_INVALID_VALUE, "field is not finite");
    if (2 * N > sbg_max_n(SBG_PRECISION_FP64))
        throw Error(SBG_ERR_UNSUPPORTED, "2 x n_sites = " + std::to_string(2 * N) + " above the solver's largest n");
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) throw Error(SBG_ERR_INVALID_VALUE, "device_id out of range");
    const size_t smem = sizeof(double2) * 2 * static_cast<size_t>(nb);
    if (smem > static_cast<size_t>(sbg::max_smem_optin()))
        throw Error(SBG_ERR_UNSUPPORTED, "n_bonds = " + std::to_string(nb) + ": the bond phases of one q exceed "
                                         "shared memory");
    DeviceGuard g(device);

    std::vector<double> half_a(2 * static_cast<size_t>(nb)), half_b(2 * static_cast<size_t>(nb));
    std::vector<double> onsite(N, 0.0), posv(3 * static_cast<size_t>(N), 0.0);
    EntryLists P(N), Q(N);
    for (int k = 0; k < nb; ++k) {
        const int i = sites[2 * k], j = sites[2 * k + 1];
        if (i < 0 || i >= N || j < 0 || j >= N)
            throw Error(SBG_ERR_INVALID_VALUE, "bond " + std::to_string(k) + ": site index out of range");
        for (int t = 0; t < 5; ++t)
            if (!std::isfinite(coef[5 * k + t])) throw Error(SBG_ERR_INVALID_VALUE, "bond " + std::to_string(k) +
                                                                                     ": coefficient not finite");
        for (int t = 0; t < 3; ++t)
            if (!std::isfinite(disp[3 * k + t])) throw Error(SBG_ERR_INVALID_VALUE, "bond " + std::to_string(k) +
                                                                                     ": displacement not finite");
        half_a[2 * k] = 0.5 * coef[5 * k];
        half_a[2 * k + 1] = 0.5 * coef[5 * k + 1];
        half_b[2 * k] = 0.5 * coef[5 * k + 2];
        half_b[2 * k + 1] = 0.5 * coef[5 * k + 3];
        P.add(i + N * j, k << 1);            // P_ij += a/2 e^{iqd}
        P.add(j + N * i, (k << 1) | 1);      // P_ji += conj(a/2 e^{iqd})
        Q.add(i + N * j, k);
        Q.add(j + N * i, k);
    }
    // On-site terms in bond order, as accumulated per site.
    for (int k = 0; k < nb; ++k) {
        const int i = sites[2 * k], j = sites[2 * k + 1];
        onsite[i] -= 0.5 * coef[5 * k + 4];
        onsite[j] -= 0.5 * coef[5 * k + 4];
    }
    if (pos) {
        for (size_t t = 0; t < posv.size(); ++t) {
            if (!std::isfinite(pos[t])) throw Error(SBG_ERR_INVALID_VALUE, "site position not finite");
            posv[t] = pos[t];
        }
    }
    P.finish();
    Q.finish();

    // One allocation: doubles (a/2, b/2, d, onsite, r), then ints (maps, ptrs, lists).
    const size_t nd = half_a.size() + half_b.size() + 3 * static_cast<size_t>(nb) + onsite.size() + posv.size();
    const size_t ni = P.map.size() + P.ptr.size() + P.list.size() + Q.map.size() + Q.ptr.size() + Q.list.size() +
                      P.ent.size() + Q.ent.size();
    std::vector<unsigned char> host(8 * nd + 4 * ni);
    std::unique_ptr<sbg_spinwave> m(new sbg_spinwave);
    m->device = device;
    m->N = N;
    m->nb = nb;
    check_cuda(cudaMalloc(&m->d_tables, host.size() + 16), "cudaMalloc(spin-wave tables)");
    unsigned char* dev = static_cast<unsigned char*>(m->d_tables);
    size_t off = 0;
    auto put = [&](const void* src, size_t bytes) {
        if (bytes) std::memcpy(host.data() + off, src, bytes);
        const void* d = dev + off;
        off += bytes;
        return d;
    };
    SwTables& T = m->T;
    T.N = N;
    T.nb = nb;
    T.field = field;
    T.half_a = static_cast<const double2*>(put(half_a.data(), 8 * half_a.size()));
    T.half_b = static_cast<const double2*>(put(half_b.data(), 8 * half_b.size()));
    T.disp = static_cast<const double*>(put(disp, 24 * static_cast<size_t>(nb)));
    T.onsite = static_cast<const double*>(put(onsite.data(), 8 * onsite.size()));
    T.pos = static_cast<const double*>(put(posv.data(), 8 * posv.size()));
    T.mapP = static_cast<const int*>(put(P.map.data(), 4 * P.map.size()));
    T.ptrP = static_cast<const int*>(put(P.ptr.data(), 4 * P.ptr.size()));
    T.listP = static_cast<const int*>(put(P.list.data(), 4 * P.list.size()));
    T.mapQ = static_cast<const int*>(put(Q.map.data(), 4 * Q.map.size()));
    T.ptrQ = static_cast<const int*>(put(Q.ptr.data(), 4 * Q.ptr.size()));
    T.listQ = static_cast<const int*>(put(Q.list.data(), 4 * Q.list.size()));
    T.entP = static_cast<const int*>(put(P.ent.data(), 4 * P.ent.size()));
    T.entQ = static_cast<const int*>(put(Q.ent.data(), 4 * Q.ent.size()));
    T.nP = static_cast<int>(P.ent.size());
    T.nQ = static_cast<int>(Q.ent.size());
    check_cuda(cudaMemcpy(m->d_tables, host.data(), host.size(), cudaMemcpyHostToDevice), "H2D spin-wave tables");
    m->assemble_smem = smem;
    if (smem > 48 * 1024)      // the attribute is per kernel and device (this one is current)
        sbg::set_smem_limit(reinterpret_cast<const void*>(k_sw_assemble), g_assemble_attr, static_cast<int>(smem));
    *out = m.release();
}

inline const double2* c2(const cuDoubleComplex* p) { return reinterpret_cast<const double2*>(p); }
inline double2* c2(cuDoubleComplex* p) { return reinterpret_cast<double2*>(p); }

}  // namespace

extern "C" {

int sbg_spinwave_create(int n_sites, int n_bonds, const int* sites, const double* coef, const double* disp,
                        const double* pos, double field, int device_id, sbg_spinwave** out) {
    return guarded([&] { create_spinwave(n_sites, n_bonds, sites, coef, disp, pos, field, device_id, out); });
}

int sbg_spinwave_destroy(sbg_spinwave* m) {
    return guarded([&] { delete m; });
}

int sbg_spinwave_matrix_size(const sbg_spinwave* m) { return m ? 2 * m->N : 0; }

int sbg_spinwave_assemble(sbg_spinwave* m, const double* d_q, int nq, cuDoubleComplex* d_A, cuDoubleComplex* d_B,
                          cudaStream_t stream) {
    return guarded([&] {
        if (!m) throw Error(SBG_ERR_INVALID_VALUE, "model == NULL");
        if (nq < 0) throw Error(SBG_ERR_INVALID_VALUE, "nq < 0");
        if (nq > 0 && (!d_q || !d_B)) throw Error(SBG_ERR_INVALID_VALUE, "null device pointer");
        DeviceGuard g(m->device);
        m->assemble(d_q, nq, c2(d_A), c2(d_B), stream);
    });
}

int sbg_spinwave_intensities(sbg_spinwave* m, const double* d_q, int nq, const double* d_W,
                             const cuDoubleComplex* d_X, const int* d_info, double* d_I, cudaStream_t stream) {
    return guarded([&] {
        if (!m) throw Error(SBG_ERR_INVALID_VALUE, "model == NULL");
        if (nq < 0) throw Error(SBG_ERR_INVALID_VALUE, "nq < 0");
        if (nq > 0 && (!d_q || !d_W || !d_X || !d_info || !d_I)) throw Error(SBG_ERR_INVALID_VALUE, "null device pointer");
        DeviceGuard g(m->device);
        m->intensities(d_q, nq, d_W, c2(d_X), d_info, d_I, stream);
    });
}

int sbg_spinwave_solve(sbg_spinwave* m, sbg_solver* s, const double* d_q, int nq, double* d_W,
                       cuDoubleComplex* d_X, double* d_I, int* d_info, cudaStream_t stream) {
    return guarded([&] {
        if (!m) throw Error(SBG_ERR_INVALID_VALUE, "model == NULL");
        DeviceGuard g(m->device);
        m->solve(s, d_q, nq, d_W, c2(d_X), d_I, d_info, stream);
    });
}

int sbg_spinwave_solve_host(sbg_spinwave* m, sbg_solver* s, const double* h_q, int nq, double* h_W,
                            cuDoubleComplex* h_X, double* h_I, int* h_info, int chunk_size, int num_streams) {
    return guarded([&] {
        if (!m) throw Error(SBG_ERR_INVALID_VALUE, "model == NULL");
        DeviceGuard g(m->device);
        m->solve_host(s, h_q, nq, h_W, c2(h_X), h_I, h_info, chunk_size, num_streams);
    });
}

}  // extern "C"
