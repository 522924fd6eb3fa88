// dev.cuh -- device helpers shared by the sm_100a kernels: element traits, parity,
// phase application from fixed-point turns, bounded mbarrier waits, and the TMA
// bulk-copy PTX (cp.async.bulk, no multicast).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace zxh {

constexpr int kThreads = 256;
constexpr uint32_t kErrTimeout = 6;  // ZXH_ERR_TIMEOUT

template <typename E>
struct ET;
template <>
struct ET<float2> {
    using R = float;
    using VT = float4;           // one 16-byte vector
    static constexpr int V = 2;  // elements per 16-byte vector
};
template <>
struct ET<double2> {
    using R = double;
    using VT = double2;
    static constexpr int V = 1;
};

// Element v of a 16-byte vector.
__device__ __forceinline__ float2 vget(const float4 &x, int v) { return v ? make_float2(x.z, x.w) : make_float2(x.x, x.y); }
__device__ __forceinline__ void vset(float4 &x, int v, float2 a)
{
    if (v) { x.z = a.x; x.w = a.y; } else { x.x = a.x; x.y = a.y; }
}
__device__ __forceinline__ float2 vget(const float2 &x, int) { return x; }
__device__ __forceinline__ void vset(float2 &x, int, float2 a) { x = a; }
__device__ __forceinline__ double2 vget(const double2 &x, int) { return x; }
__device__ __forceinline__ void vset(double2 &x, int, double2 a) { x = a; }

// exp(2 pi i th / 2^64) from a 1024-entry table (top 10 bits of th) and a short
// Taylor series for the rest (angle below 2 pi / 1024): truncation error below
// 1e-13 in float, below 1e-19 in double.
__device__ __forceinline__ float2 phase_factor(const float2 *tab, int64_t th)
{
    const uint64_t u = static_cast<uint64_t>(th);
    const float2 t = tab[u >> 54];
    const float eps = __ull2float_rn(u & ((1ULL << 54) - 1ULL)) * 3.4061215800865545e-19f;  // 2 pi / 2^64
    const float e2 = eps * eps;
    const float s = fmaf(-eps * e2, 0.16666667f, eps);
    const float c = fmaf(-0.5f, e2, 1.0f);
    return make_float2(t.x * c - t.y * s, t.x * s + t.y * c);
}

// exp(2 pi i th / 2^32) for complex64 amplitudes: the same 1024-entry table for
// the top 10 bits of a 32-bit turn count, and a third-order Taylor step for the
// low 22 bits (angle below 2 pi / 1024; truncation error below 1e-12). The low
// bits become a float without a conversion instruction: they are placed in the
// mantissa of 1.0f.
__device__ __forceinline__ float2 phase_factor32(const float2 *tab, uint32_t th)
{
    const float2 t = tab[th >> 22];
    const float f = __uint_as_float(0x3F800000u | ((th << 1) & 0x007FFFFEu));  // 1 + low22 / 2^22
    const float eps = fmaf(f, 6.1359231515425650e-3f, -6.1359231515425650e-3f);  // low22 * 2 pi / 2^32
    const float e2 = eps * eps;
    const float s = fmaf(-eps * e2, 0.16666667f, eps);
    const float c = fmaf(-0.5f, e2, 1.0f);
    return make_float2(t.x * c - t.y * s, t.x * s + t.y * c);
}

// Nearest 32-bit turn count of a 64-bit one (both modulo a full turn).
__device__ __forceinline__ uint32_t turns32(int64_t th)
{
    return static_cast<uint32_t>((static_cast<uint64_t>(th) + 0x80000000ULL) >> 32);
}

__device__ __forceinline__ double2 phase_factor(const double2 *tab, int64_t th)
{
    const uint64_t u = static_cast<uint64_t>(th);
    const double2 t = tab[u >> 54];
    const double eps = __ull2double_rn(u & ((1ULL << 54) - 1ULL)) * 3.4061215800865545e-19;
    const double e2 = eps * eps;
    const double s = eps * (1.0 - e2 * (1.0 / 6.0) * (1.0 - e2 * (1.0 / 20.0)));
    const double c = 1.0 - e2 * 0.5 * (1.0 - e2 * (1.0 / 12.0) * (1.0 - e2 * (1.0 / 30.0)));
    return make_double2(t.x * c - t.y * s, t.x * s + t.y * c);
}

// a * x + b * y for real a, b: complex64 amplitudes as (re, im) pairs take paired
// FP32 FMAs (two lanes of work per instruction).
__device__ __forceinline__ float2 rmad2(float a, float2 x, float b, float2 y)
{
    return __ffma2_rn(make_float2(b, b), y, __fmul2_rn(make_float2(a, a), x));
}
__device__ __forceinline__ double2 rmad2(double a, double2 x, double b, double2 y)
{
    return make_double2(fma(b, y.x, a * x.x), fma(b, y.y, a * x.y));
}

template <typename E>
__device__ __forceinline__ E cmul(E a, E b)
{
    E o;
    o.x = a.x * b.x - a.y * b.y;
    o.y = a.x * b.y + a.y * b.x;
    return o;
}

// Trailing zeros of a compile-time constant (index arithmetic in unrolled loops).
// Trailing zeros of x > 0. Not recursive, so it is inlined and, inside a fully
// unrolled loop, folds to a constant (register arrays indexed by it then stay in
// registers; a recursive form stays a call and forces them into local memory).
__host__ __device__ __forceinline__ constexpr int ctz_const(int x)
{
    int n = 0;
    while (n < 31 && !((x >> n) & 1)) n++;
    return n;
}

__device__ __forceinline__ int par64(uint64_t x) { return __popcll(x) & 1; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Multiplies a by exp(i * 2 pi * th / 2^64). th is a signed fixed-point number of
// turns, so the angle is pi * x with x = th / 2^63 in [-1, 1).
__device__ __forceinline__ float2 apply_phase(float2 a, int64_t th)
{
    // x = xh + xl: xh has the top 24 bits (exact in float), xl < 2^-23 the rest.
    const int32_t hi = static_cast<int32_t>(th >> 40);
    const float xh = static_cast<float>(hi) * 0x1p-23f;
    const float xl = static_cast<float>(static_cast<uint64_t>(th) & ((1ULL << 40) - 1ULL)) * 0x1p-63f;
    float s, c;
    sincospif(xh, &s, &c);
    // first-order correction for xl (second-order term below 1e-13)
    const float d = 3.14159265358979f * xl;
    const float s2 = fmaf(d, c, s), c2 = fmaf(-d, s, c);
    float2 o;
    o.x = a.x * c2 - a.y * s2;
    o.y = a.x * s2 + a.y * c2;
    return o;
}

__device__ __forceinline__ double2 apply_phase(double2 a, int64_t th)
{
    const double x = static_cast<double>(th) * 0x1p-63;
    double s, c;
    sincospi(x, &s, &c);
    double2 o;
    o.x = a.x * c - a.y * s;
    o.y = a.x * s + a.y * c;
    return o;
}

__device__ __forceinline__ int64_t warp_sum_i64(int64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_f64(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct DevStatusView { uint32_t code; uint32_t where; uint64_t info; };

__device__ __forceinline__ void report(void *status, uint32_t code, uint32_t where, uint64_t info)
{
    DevStatusView *s = static_cast<DevStatusView *>(status);
    if (atomicCAS(&s->code, 0u, code) == 0u) {
        s->where = where;
        s->info = info;
    }
}

// ---- mbarrier ----

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barrier `id` over `count` threads (a multiple of 32), with an OR of pred
// across them (bar.red.or).
__device__ __forceinline__ bool named_barrier_or(int id, int count, bool pred)
{
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"(uint32_t(pred)), "r"(id), "r"(count)
        : "memory");
    return out != 0;
}

__device__ __forceinline__ void named_barrier(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity; gives up after about 2^31 SM clocks
// (around a second) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1LL << 31)) return false;
    return true;
}

// ---- TMA bulk copies (1-D, no tensor map, no multicast) ----

__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_s2g(void *gdst, const void *smem_src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(smem_src)),
                 "r"(bytes)
                 : "memory");
}

// Asks L2 to fetch [gsrc, gsrc + bytes) from memory (no destination, nothing to
// wait for); both 16-byte aligned.
__device__ __forceinline__ void bulk_prefetch_l2(const void *gsrc, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gsrc), "r"(bytes) : "memory");
}

// 16-byte asynchronous copy global -> shared through L2 (cp.async.cg); both
// addresses 16-byte aligned. A thread's copies complete in commit groups.
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// waits until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace zxh
