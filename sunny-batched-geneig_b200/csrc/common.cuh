// Device helpers shared by every stage kernel: complex arithmetic on the
// interleaved (re, im) layout of cuDoubleComplex / cuFloatComplex, team
// reductions, and the sm_100a bulk-copy (TMA) + mbarrier primitives used to
// stage matrices into shared memory.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace sbg {

// ----------------------------------------------------------------------------- complex

template <typename R> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float>  { using type = float2; };
template <typename R> using cplx = typename cplx_t<R>::type;

template <typename R> __device__ __forceinline__ cplx<R> mk(R re, R im) { cplx<R> z; z.x = re; z.y = im; return z; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }
// a * b
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// conj(a) * b
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
// acc + a * b
template <typename C> __device__ __forceinline__ C cfma(C a, C b, C acc) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc - a * b
template <typename C> __device__ __forceinline__ C cfms(C a, C b, C acc) {
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
// acc + conj(a) * b
template <typename C> __device__ __forceinline__ C cfmac(C a, C b, C acc) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
// acc - a * conj(b)
template <typename C> __device__ __forceinline__ C cfmsc(C a, C b, C acc) {
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);  acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
template <typename C> __device__ __forceinline__ auto cabs2(C a) -> decltype(a.x) { return a.x * a.x + a.y * a.y; }

template <typename R> __device__ __forceinline__ R shfl_xor(R v, int m, int width = 32) {
    return __shfl_xor_sync(0xffffffffu, v, m, width);
}
template <typename C> __device__ __forceinline__ C cshfl(C v, int src, int width = 32) {
    v.x = __shfl_sync(0xffffffffu, v.x, src, width);
    v.y = __shfl_sync(0xffffffffu, v.y, src, width);
    return v;
}
template <typename R> __device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += shfl_xor(v, m);
    return v;
}
template <typename R> __device__ __forceinline__ R group_sum(R v, int width) {
    for (int m = width >> 1; m >= 1; m >>= 1) v += shfl_xor(v, m, width);
    return v;
}

// Leading dimension for an n x n tile of 16- or 8-byte elements in shared memory:
// odd, so a warp walking a row (stride ld) touches distinct banks, and never 7 mod 8,
// where a walk along a diagonal (stride ld + 1 complex = a multiple of 128 bytes)
// would put every lane in the same bank.
__host__ __device__ __forceinline__ int tile_ld(int n) {
    int ld = n | 1;
    if ((ld & 7) == 7) ld += 2;
    return ld;
}

// ----------------------------------------------------------------------------- bulk copy

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// Returns true once the phase with the given parity has completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait: gives up after max_polls polls and returns false (never spins forever).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_polls) {
    for (uint32_t i = 0; i < max_polls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Global -> shared bulk copy (cp.async.bulk, no multicast), completion signalled on bar.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

constexpr uint32_t kMaxPolls = 1u << 24;   // far beyond any real copy; a timeout is reported, not hung on

// Status bits written to the per-pair info word when something other than the
// LAPACK conventions happens (kept above any n + i value).
constexpr int kInfoCopyTimeout = 1 << 29;

// ----------------------------------------------------------------------------- reciprocal

// 1/u by Newton-Raphson iteration for the reciprocal (the textbook method: each step
// r <- r + r (1 - u r) squares the relative error) from the hardware reciprocal estimate
// (rcp.approx.ftz.f64); two steps.  Used by the inverse iteration's factorization, where it is
// shorter than a correctly rounded division in the dependent chain and no correct rounding is
// needed (every vector's residual is checked); |u| >= eps ||T|| there keeps u normal.
// sbg_selftest_reciprocal exposes it so a test can compare it with the correctly rounded 1.0 / u.
__device__ __forceinline__ double recip_nr(double u) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(u));
    double e = fma(-u, r, 1.0);
    r = fma(r, e, r);
    e = fma(-u, r, 1.0);
    return fma(r, e, r);
}

}  // namespace sbg
