// sampler.cu -- multinomial sampler of the B200-native ZXH path (sm_100a).
//
// Draws the same outcomes as the reference GPU sampler when fed the same seed: it
// consumes the reference's uniform stream (splitmix64 of seed-mixed shot and output
// indices, src/zxh/src/measure/measure_cuda.cu:387-443,493-515) with the same two-
// level structure (segments of 2^12 amplitudes, then an offset inside the segment),
// and returns shots grouped by segment in the reference's output order. The
// machinery is new:
//   seg_mass_kernel      one streaming read of the state: per-segment FP64 |amp|^2
//                        mass, one warp per segment (and the 32 lane-range masses of
//                        each segment, kept for the resolve step).
//   mass scan (3 kernels) inclusive FP64 scan of the masses: the segment CDF (the
//                        reference runs segment_mass_kernel + a CUB scan).
//   count_kernel         shot -> segment by binary search, warp-aggregated atomics.
//   offsets (3 kernels)  exclusive scan of the per-segment counts.
//   resolve_warp_kernel  segments hit by <= 32 shots: one warp streams the segment
//                        once, lane-scans it and places each shot with a warp-
//                        cooperative search (ballot over lane prefixes, then over
//                        4-amplitude sub-ranges).
//   resolve_cta_kernel   heavier segments, one per CTA (round robin): the CTA builds
//                        the segment CDF in shared memory and binary-searches it.
//   map_kernel           real index -> packed virtual bits (measure_cuda.cu:315-338).
// No kernel waits on another CTA.
#include "core.h"
#include "dev.cuh"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

constexpr uint64_t kSeedShot = 0x510e527fade682d1ULL;    // measure_cuda.cu:427
constexpr uint64_t kSeedOffset = 0x9b05688c2b3e6c1fULL;  // measure_cuda.cu:499
constexpr int kWarpMax = 32;
constexpr int kScanBlock = 4096;

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    uint64_t z = x + 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// (mant + 1) / (2^53 + 1) evaluated in double; 2^53 + 1 rounds to 2^53 as on the
// reference device (measure_cuda.cu:395-410).
__device__ __forceinline__ double uniform_open01(uint64_t seed)
{
    const uint64_t mant = splitmix64(seed) >> 11;
    return (static_cast<double>(mant) + 1.0) / (static_cast<double>(1ULL << 53) + 1.0);
}

template <typename E>
__device__ __forceinline__ double prob(const E &a)
{
    const double re = double(a.x), im = double(a.y);
    return re * re + im * im;
}


// |amp|^2 mass of seg[lo, hi), in order; complex64 ranges with even bounds use
// 16-byte loads.
__device__ __forceinline__ double range_mass(const float2 *seg, uint32_t lo, uint32_t hi)
{
    double part = 0.0;
    if (!((lo | hi) & 1)) {
        const float4 *v = reinterpret_cast<const float4 *>(seg);
        for (uint32_t k = lo / 2; k < hi / 2; k++) {
            const float4 x = __ldg(v + k);
            part += double(x.x) * x.x + double(x.y) * x.y;
            part += double(x.z) * x.z + double(x.w) * x.w;
        }
        return part;
    }
    for (uint32_t k = lo; k < hi; k++) part += prob(seg[k]);
    return part;
}

__device__ __forceinline__ double range_mass(const double2 *seg, uint32_t lo, uint32_t hi)
{
    double part = 0.0;
    for (uint32_t k = lo; k < hi; k++) part += prob(__ldg(seg + k));
    return part;
}

// ---------------------------------------------------------------------------

// Mass of lane l's range [l p, (l + 1) p) of a full 4096-amplitude segment, p =
// 128, read coalesced: in step g the warp reads 32 consecutive 16-byte vectors,
// which all belong to range g / G (G steps per range), and the range's mass is
// the warp's sum of them; lane l keeps range l. The same code runs in the segment
// pass and in the resolve step's fallback, so both see the same numbers.
__device__ __forceinline__ double vec_mass(const float4 &x)
{
    return (double(x.x) * x.x + double(x.y) * x.y) + (double(x.z) * x.z + double(x.w) * x.w);
}
__device__ __forceinline__ double vec_mass(const double2 &x) { return x.x * x.x + x.y * x.y; }

template <typename E>
__device__ __forceinline__ double lane_range_mass(const E *seg, int lane)
{
    using VT = typename ET<E>::VT;
    constexpr int G = 4096 / ET<E>::V / 32 / 32;  // steps per range: 2 (complex64), 4 (complex128)
    const VT *v = reinterpret_cast<const VT *>(seg);
    double mine = 0.0;
#pragma unroll 4
    for (int r = 0; r < 32; r++) {
        VT x[G];
#pragma unroll
        for (int i = 0; i < G; i++) x[i] = __ldcs(v + (r * G + i) * 32 + lane);
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < G; i++) t += vec_mass(x[i]);
        t = warp_sum_f64(t);
        if (lane == r) mine = t;
    }
    return mine;
}

// Lane l of a warp owns amplitudes [l p, (l + 1) p) of a segment, p = seglen / 32
// rounded up; its mass and the warp's inclusive prefix over lanes. The segment
// kernel and the resolve kernel both use this order, so a segment's total and its
// lane prefixes are the same numbers in both.
__device__ __forceinline__ double lane_prefix(double part, int lane)
{
    double incl = part;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    return incl;
}

// Per-segment FP64 mass, one warp per segment: one streaming read of the state.
// With parts, every lane's range mass is kept for the resolve step.
template <typename E>
__global__ void __launch_bounds__(kThreads) seg_mass_kernel(const E *__restrict__ state, uint64_t nseg, uint32_t seglen,
                                                            double *__restrict__ mass, double *__restrict__ parts)
{
    const int lane = threadIdx.x & 31;
    const uint64_t w0 = (uint64_t(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    const uint64_t nw = (uint64_t(gridDim.x) * kThreads) >> 5;
    const uint32_t per_lane = (seglen + 31) / 32;
    const uint32_t lo = min(seglen, uint32_t(lane) * per_lane), hi = min(seglen, lo + per_lane);
    for (uint64_t sg = w0; sg < nseg; sg += nw) {
        const double part = seglen == 4096 ? lane_range_mass(state + sg * seglen, lane)
                                           : range_mass(state + sg * seglen, lo, hi);
        if (parts) parts[sg * 32 + uint64_t(lane)] = part;
        const double total = __shfl_sync(0xffffffffu, lane_prefix(part, lane), 31);
        if (lane == 0) mass[sg] = total;
    }
}

__device__ __forceinline__ uint64_t upper_index(const double *cdf, uint64_t n, double tau)
{
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] <= tau) lo = mid + 1;
        else hi = mid;
    }
    return lo >= n ? n - 1 : lo;
}

__global__ void __launch_bounds__(kThreads) count_kernel(const double *__restrict__ segcdf, uint64_t nseg,
                                                         uint64_t stream_seed, uint64_t shots,
                                                         unsigned long long *__restrict__ counts)
{
    const double total = segcdf[nseg - 1];
    for (uint64_t base = uint64_t(blockIdx.x) * kThreads; base < shots; base += uint64_t(gridDim.x) * kThreads) {
        const uint64_t idx = base + threadIdx.x;
        const bool live = idx < shots && total > 0.0;
        uint64_t seg = ~0ULL;
        if (live) {
            const double u = uniform_open01(stream_seed ^ (kSeedShot + idx));
            seg = upper_index(segcdf, nseg, u * total);
        }
        // one atomic per distinct segment in the warp
        const unsigned peers = __match_any_sync(0xffffffffu, seg);
        const int leader = __ffs(peers) - 1;
        if (live && int(threadIdx.x & 31) == leader) atomicAdd(&counts[seg], static_cast<unsigned long long>(__popc(peers)));
    }
}

// exclusive scan of counts: block sums, scan of block sums, block scans
// Scan of n values in blocks of kScanBlock: per-block sums, one small scan over
// them, then each block's scan plus its offset. T = unsigned long long for the
// shot counts (exclusive offsets), double for the segment masses (inclusive CDF,
// written over the masses).
template <typename T>
__global__ void __launch_bounds__(kThreads) block_sum_kernel(const T *__restrict__ v, uint64_t n, T *__restrict__ bsum)
{
    __shared__ T sh[kThreads / 32];
    const uint64_t b0 = uint64_t(blockIdx.x) * kScanBlock;
    T acc = 0;
    for (uint64_t i = b0 + threadIdx.x; i < (n < b0 + kScanBlock ? n : b0 + kScanBlock); i += kThreads) acc += v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        T t = 0;
        for (int w = 0; w < kThreads / 32; w++) t += sh[w];
        bsum[blockIdx.x] = t;
    }
}

template <typename T>
__global__ void scan_small_kernel(T *v, uint64_t n)
{
    // single thread, exclusive; n is at most a few thousand block sums
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    T run = 0;
    for (uint64_t i = 0; i < n; i++) {
        const T x = v[i];
        v[i] = run;
        run += x;
    }
}

// in and out may be the same array (every thread reads its own values first)
template <typename T, bool INCL>
__global__ void __launch_bounds__(kThreads) block_scan_kernel(const T *in, uint64_t n, const T *__restrict__ boff,
                                                              T *out)
{
    constexpr int PER = kScanBlock / kThreads;  // 16 consecutive values per thread
    __shared__ T sh[kThreads];
    const uint64_t b0 = uint64_t(blockIdx.x) * kScanBlock + uint64_t(threadIdx.x) * PER;
    T loc[PER];
    T acc = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        loc[k] = (b0 + k < n) ? in[b0 + k] : T(0);
        acc += loc[k];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
        const T x = threadIdx.x >= unsigned(o) ? sh[threadIdx.x - o] : T(0);
        __syncthreads();
        sh[threadIdx.x] += x;
        __syncthreads();
    }
    T run = boff[blockIdx.x] + (sh[threadIdx.x] - acc);
#pragma unroll
    for (int k = 0; k < PER; k++) {
        if (INCL) run += loc[k];
        if (b0 + k < n) out[b0 + k] = run;
        if (!INCL) run += loc[k];
    }
}

// segments hit by at most kWarpMax shots
template <typename E>
__global__ void __launch_bounds__(kThreads) resolve_warp_kernel(const E *__restrict__ state, uint64_t nseg,
                                                                uint32_t seglen, const unsigned long long *counts,
                                                                const unsigned long long *offsets, uint64_t stream2,
                                                                uint64_t *__restrict__ real_out,
                                                                uint32_t *heavy_list, uint32_t *heavy_count,
                                                                const double *__restrict__ parts)
{
    const int lane = threadIdx.x & 31;
    const uint64_t gwarp = (uint64_t(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * kThreads) >> 5;
    const uint32_t per_lane = (seglen + 31) / 32;  // amplitudes owned by a lane
    for (uint64_t g0 = gwarp * 32; g0 < nseg; g0 += nwarps * 32) {
        const uint64_t gl = g0 + uint64_t(lane);
        const unsigned long long cl = gl < nseg ? counts[gl] : 0ULL;
        unsigned todo = __ballot_sync(0xffffffffu, cl != 0);
        if (cl > kWarpMax) heavy_list[atomicAdd(heavy_count, 1u)] = uint32_t(gl);
        todo &= __ballot_sync(0xffffffffu, cl <= kWarpMax);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint64_t g = g0 + uint64_t(src);
            const unsigned long long cnt = __shfl_sync(0xffffffffu, cl, src);
            const unsigned long long off = offsets[g];
            const E *seg = state + g * seglen;
            // lane range [lane*per_lane, (lane+1)*per_lane): its mass from the
            // segment kernel when kept, else read again
            const uint32_t lo = min(seglen, uint32_t(lane) * per_lane);
            const uint32_t hi = min(seglen, lo + per_lane);
            const double part = parts ? parts[g * 32 + uint64_t(lane)]
                                      : seglen == 4096 ? lane_range_mass(seg, lane) : range_mass(seg, lo, hi);
            const double incl = lane_prefix(part, lane);
            const double total = __shfl_sync(0xffffffffu, incl, 31);
            const double excl = incl - part;
            // this lane's shot
            double tau = 0.0;
            if (uint64_t(lane) < cnt) tau = uniform_open01(stream2 ^ (kSeedOffset + off + uint64_t(lane))) * total;
            if (seglen == 4096) {
                // full segments: the owner range is 128 amplitudes, 4 per lane; they
                // are loaded at once and kept in registers, and the next shot's are
                // on their way while this shot is placed (the sums run in the same
                // order as the general path below, so the draws are the same)
                E cur[4], nxt[4];
                double t = __shfl_sync(0xffffffffu, tau, 0);
                int owner = __popc(__ballot_sync(0xffffffffu, incl <= t));
                if (owner < 32) {
#pragma unroll
                    for (int i = 0; i < 4; i++) cur[i] = __ldg(seg + uint32_t(owner) * 128u + uint32_t(lane) * 4u + i);
                }
#pragma unroll 1
                for (int j = 0; j < int(cnt); j++) {
                    double tn = 0.0;
                    int on = 32;
                    if (j + 1 < int(cnt)) {
                        tn = __shfl_sync(0xffffffffu, tau, j + 1);
                        on = __popc(__ballot_sync(0xffffffffu, incl <= tn));
                        if (on < 32) {
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                nxt[i] = __ldg(seg + uint32_t(on) * 128u + uint32_t(lane) * 4u + i);
                        }
                    }
                    uint64_t hit = seglen - 1;
                    if (owner < 32) {
                        const double obase = __shfl_sync(0xffffffffu, excl, owner);
                        double p[4], sp = 0.0;
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            p[i] = prob(cur[i]);
                            sp += p[i];
                        }
                        double sincl = sp;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const double v = __shfl_up_sync(0xffffffffu, sincl, o);
                            if (lane >= o) sincl += v;
                        }
                        const int sl = __popc(__ballot_sync(0xffffffffu, obase + sincl <= t));
                        uint32_t found = 4;  // past this lane's sub-range
                        if (sl < 32 && lane == sl) {
                            double run = obase + sincl - sp;
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                run += p[i];
                                if (found == 4 && run > t) found = uint32_t(i);
                            }
                        }
                        const uint32_t fs = __shfl_sync(0xffffffffu, found, sl < 32 ? sl : 0);
                        hit = uint64_t(owner) * 128u + (sl < 32 ? uint32_t(sl) * 4u + fs : 128u);
                        if (hit >= seglen) hit = seglen - 1;
                    }
                    if (lane == 0) real_out[off + uint64_t(j)] = g * seglen + hit;
                    t = tn;
                    owner = on;
#pragma unroll
                    for (int i = 0; i < 4; i++) cur[i] = nxt[i];
                }
                continue;
            }
            for (int j = 0; j < int(cnt); j++) {
                const double t = __shfl_sync(0xffffffffu, tau, j);
                // owner lane: first lane whose inclusive prefix exceeds t
                const unsigned le = __ballot_sync(0xffffffffu, incl <= t);
                int owner = __popc(le);
                uint64_t hit;
                if (owner >= 32) {
                    hit = seglen - 1;
                } else {
                    // cooperative search in the owner's range: each lane takes a sub-range
                    const double obase = __shfl_sync(0xffffffffu, excl, owner);
                    const uint32_t olo = uint32_t(owner) * per_lane;
                    const uint32_t ohi = min(seglen, olo + per_lane);
                    const uint32_t sub = (per_lane + 31) / 32;
                    const uint32_t slo = min(ohi, olo + uint32_t(lane) * sub);
                    const uint32_t shi = min(ohi, slo + sub);
                    double sp = 0.0;
                    for (uint32_t k = slo; k < shi; k++) sp += prob(seg[k]);
                    double sincl = sp;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const double v = __shfl_up_sync(0xffffffffu, sincl, o);
                        if (lane >= o) sincl += v;
                    }
                    const unsigned le2 = __ballot_sync(0xffffffffu, obase + sincl <= t);
                    const int sl = __popc(le2);
                    uint32_t found = ohi;  // none below the end of the owner's range
                    if (sl < 32 && lane == sl) {
                        double run = obase + sincl - sp;
                        found = shi;
                        for (uint32_t k = slo; k < shi; k++) {
                            run += prob(seg[k]);
                            if (run > t) {
                                found = k;
                                break;
                            }
                        }
                    }
                    const uint32_t fs = __shfl_sync(0xffffffffu, found, sl < 32 ? sl : 0);
                    hit = (sl < 32) ? fs : ohi;
                    if (hit >= seglen) hit = seglen - 1;
                }
                if (lane == 0) real_out[off + uint64_t(j)] = g * seglen + hit;
            }
        }
    }
}

// Shared CDF of a heavy segment: entry k at k + k / 16, so the 16 consecutive
// entries a thread scans sit in distinct banks across the warp.
__device__ __forceinline__ uint32_t cdf_slot(uint32_t k) { return k + (k >> 4); }

__device__ __forceinline__ uint64_t upper_index_padded(const double *cdf, uint64_t n, double tau)
{
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (cdf[cdf_slot(uint32_t(mid))] <= tau) lo = mid + 1;
        else hi = mid;
    }
    return lo >= n ? n - 1 : lo;
}

template <typename E>
__global__ void __launch_bounds__(kThreads) resolve_cta_kernel(const E *__restrict__ state, uint32_t seglen,
                                                               const unsigned long long *counts,
                                                               const unsigned long long *offsets, uint64_t stream2,
                                                               uint64_t *__restrict__ real_out,
                                                               const uint32_t *heavy_list,
                                                               const uint32_t *heavy_count)
{
    extern __shared__ double cdf[];  // cdf_slot(seglen) entries
    __shared__ double s_warp[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nh = *heavy_count;
    // heavy segment h goes to CTA h mod grid, which places all of its shots
    for (uint32_t h = blockIdx.x; h < nh; h += gridDim.x) {
        const uint64_t g = heavy_list[h];
        const unsigned long long cnt = counts[g], off = offsets[g];
        // build the segment CDF once for all of its shots: coalesced loads, a serial
        // scan of each thread's consecutive range, a block scan of the range totals
        const E *seg = state + g * seglen;
        const uint32_t per = (seglen + kThreads - 1) / kThreads;
        const uint32_t lo = min(seglen, threadIdx.x * per), hi = min(seglen, lo + per);
        for (uint32_t k = threadIdx.x; k < seglen; k += kThreads) cdf[cdf_slot(k)] = prob(__ldg(seg + k));
        __syncthreads();
        double run = 0.0;
        for (uint32_t k = lo; k < hi; k++) {
            run += cdf[cdf_slot(k)];
            cdf[cdf_slot(k)] = run;
        }
        double incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        double add = incl - run;
        for (int w = 0; w < warp; w++) add += s_warp[w];
        for (uint32_t k = lo; k < hi; k++) cdf[cdf_slot(k)] += add;
        __syncthreads();
        const double total = cdf[cdf_slot(seglen - 1)];
        for (uint64_t j = threadIdx.x; j < cnt; j += kThreads) {
            const double tau = uniform_open01(stream2 ^ (kSeedOffset + off + j)) * total;
            real_out[off + j] = g * seglen + upper_index_padded(cdf, seglen, tau);
        }
        __syncthreads();  // cdf and s_warp are reused by the next heavy segment
    }
}

__global__ void __launch_bounds__(kThreads) map_kernel(const uint64_t *__restrict__ real, uint64_t shots,
                                                       const uint64_t *__restrict__ coltab, uint64_t b,
                                                       uint64_t *__restrict__ words)
{
    __shared__ uint64_t tab[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += kThreads) tab[i >> 8][i & 255] = coltab[i];
    __syncthreads();
    for (uint64_t i = uint64_t(blockIdx.x) * kThreads + threadIdx.x; i < shots; i += uint64_t(gridDim.x) * kThreads) {
        const uint64_t r = real[i];
        uint64_t v = b;
#pragma unroll
        for (int k = 0; k < 8; k++) v ^= tab[k][(r >> (8 * k)) & 255];
        words[i] = v;
    }
}

// ---------------------------------------------------------------------------
// Counts: the distinct outcomes of a draw and how often each came up, without
// copying the shots to the host. The draw leaves every shot's real index grouped
// by segment (segments in increasing order), so counting is per segment: a
// segment with at most kWarpMax shots sorts its offsets in one warp (bitonic
// network over the lanes) and run-length encodes them; a heavier segment (the
// sampler's heavy list) builds a histogram of its 2^12 offsets in shared memory.
// Pass 1 writes each segment's number of distinct outcomes, a scan of those gives
// every segment's first output slot, and pass 2 repeats the work and writes the
// (virtual word, count) pairs there, in increasing real index.

__device__ __forceinline__ uint32_t warp_sort32(uint32_t v, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool up = (lane & k) == 0;
            const bool low = (lane & j) == 0;
            v = (low == up) ? min(v, o) : max(v, o);
        }
    return v;
}

__device__ __forceinline__ uint64_t map_word(const uint64_t (*tab)[256], uint64_t b, uint64_t r)
{
    uint64_t v = b;
#pragma unroll
    for (int k = 0; k < 8; k++) v ^= tab[k][(r >> (8 * k)) & 255];
    return v;
}

template <bool WRITE>
__global__ void __launch_bounds__(kThreads) count_light_kernel(const uint64_t *__restrict__ real, uint64_t nseg,
                                                               uint32_t seglen, const unsigned long long *counts,
                                                               const unsigned long long *offsets,
                                                               unsigned long long *nuniq,
                                                               const unsigned long long *uoff,
                                                               const uint64_t *__restrict__ coltab, uint64_t b,
                                                               uint64_t *__restrict__ words,
                                                               uint64_t *__restrict__ hits)
{
    __shared__ uint64_t tab[WRITE ? 8 : 1][256];
    if constexpr (WRITE) {
        for (int i = threadIdx.x; i < 8 * 256; i += kThreads) tab[i >> 8][i & 255] = coltab[i];
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const uint64_t gwarp = (uint64_t(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * kThreads) >> 5;
    for (uint64_t g0 = gwarp * 32; g0 < nseg; g0 += nwarps * 32) {
        const uint64_t gl = g0 + uint64_t(lane);
        const unsigned long long cl = gl < nseg ? counts[gl] : 0ULL;
        if (!WRITE && gl < nseg && cl == 0) nuniq[gl] = 0;
        unsigned todo = __ballot_sync(0xffffffffu, cl != 0 && cl <= kWarpMax);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint64_t g = g0 + uint64_t(src);
            const uint32_t cnt = uint32_t(__shfl_sync(0xffffffffu, cl, src));
            const uint64_t base = g * seglen;
            const unsigned long long off = offsets[g];
            uint32_t key = 0xffffffffu;  // padding sorts last
            if (uint32_t(lane) < cnt) key = uint32_t(real[off + uint64_t(lane)] - base);
            key = warp_sort32(key, lane);
            const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
            const bool first = uint32_t(lane) < cnt && (lane == 0 || key != prev);
            const unsigned starts = __ballot_sync(0xffffffffu, first);
            if constexpr (!WRITE) {
                if (lane == 0) nuniq[g] = __popc(starts);
            } else if (first) {
                const unsigned above = starts & ~((2u << lane) - 1u);  // lane 31: 2u << 31 wraps to 0, nothing above
                const uint32_t next = above ? uint32_t(__ffs(above) - 1) : cnt;
                const uint64_t slot = uoff[g] + uint64_t(__popc(starts & ((1u << lane) - 1u)));
                words[slot] = map_word(tab, b, base + key);
                hits[slot] = next - uint32_t(lane);
            }
        }
    }
}

// heavy segment h goes to CTA h mod grid (shared histogram of seglen bins)
template <bool WRITE>
__global__ void __launch_bounds__(kThreads) count_heavy_kernel(const uint64_t *__restrict__ real, uint32_t seglen,
                                                               const unsigned long long *counts,
                                                               const unsigned long long *offsets,
                                                               const uint32_t *heavy_list,
                                                               const uint32_t *heavy_count,
                                                               unsigned long long *nuniq,
                                                               const unsigned long long *uoff,
                                                               const uint64_t *__restrict__ coltab, uint64_t b,
                                                               uint64_t *__restrict__ words,
                                                               uint64_t *__restrict__ hits)
{
    __shared__ uint32_t hist[4096];
    __shared__ uint32_t s_warp[kThreads / 32];
    __shared__ uint64_t tab[WRITE ? 8 : 1][256];
    if constexpr (WRITE) {
        for (int i = threadIdx.x; i < 8 * 256; i += kThreads) tab[i >> 8][i & 255] = coltab[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nh = *heavy_count;
    const uint32_t per = (seglen + kThreads - 1) / kThreads;  // bins of a thread (16 for full segments)
    for (uint32_t h = blockIdx.x; h < nh; h += gridDim.x) {
        const uint64_t g = heavy_list[h];
        const unsigned long long cnt = counts[g], off = offsets[g];
        const uint64_t base = g * seglen;
        for (uint32_t k = threadIdx.x; k < seglen; k += kThreads) hist[k] = 0;
        __syncthreads();
        for (uint64_t j = threadIdx.x; j < cnt; j += kThreads) atomicAdd(&hist[uint32_t(real[off + j] - base)], 1u);
        __syncthreads();
        const uint32_t lo = min(seglen, uint32_t(threadIdx.x) * per), hi = min(seglen, lo + per);
        uint32_t mine = 0;
        for (uint32_t k = lo; k < hi; k++) mine += hist[k] != 0;
        // block exclusive scan of the per-thread distinct counts
        uint32_t incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            before += w < warp ? s_warp[w] : 0;
            total += s_warp[w];
        }
        if constexpr (!WRITE) {
            if (threadIdx.x == 0) nuniq[g] = total;
        } else {
            uint64_t slot = uoff[g] + before + incl - mine;
            for (uint32_t k = lo; k < hi; k++)
                if (hist[k]) {
                    words[slot] = map_word(tab, b, base + k);
                    hits[slot] = hist[k];
                    slot++;
                }
        }
        __syncthreads();  // hist and s_warp are reused by the next heavy segment
    }
}

__global__ void count_total_kernel(const unsigned long long *nuniq, const unsigned long long *uoff, uint64_t nseg,
                                   unsigned long long *total)
{
    *total = uoff[nseg - 1] + nuniq[nseg - 1];
}

}  // namespace

cudaError_t run_counts(const SamplerScratch &sc, int m, uint64_t b, unsigned long long *nuniq,
                       unsigned long long *uoff, unsigned long long *total, uint64_t *words, uint64_t *hits,
                       int pass, int sms, cudaStream_t st, uint64_t &kernels)
{
    const uint64_t local = 1ULL << m;
    const uint32_t seglen = uint32_t(std::min<uint64_t>(4096, local));
    const uint64_t nseg = local / seglen;
    const uint64_t nblk = (nseg + kScanBlock - 1) / kScanBlock;
    const uint64_t warps_needed = (nseg + 31) / 32;
    const unsigned gw = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((warps_needed * 32 + kThreads - 1) / kThreads,
                                                                          uint64_t(sms) * 8)));
    const unsigned gh = unsigned(sms) * 4;
    if (pass == 1) {
        count_light_kernel<false><<<gw, kThreads, 0, st>>>(sc.real, nseg, seglen, sc.counts, sc.offsets, nuniq,
                                                           nullptr, nullptr, b, nullptr, nullptr);
        count_heavy_kernel<false><<<gh, kThreads, 0, st>>>(sc.real, seglen, sc.counts, sc.offsets, sc.heavy_list,
                                                           sc.heavy_count, nuniq, nullptr, nullptr, b, nullptr,
                                                           nullptr);
        block_sum_kernel<unsigned long long><<<unsigned(nblk), kThreads, 0, st>>>(nuniq, nseg, sc.bsum);
        scan_small_kernel<unsigned long long><<<1, 32, 0, st>>>(sc.bsum, nblk);
        block_scan_kernel<unsigned long long, false><<<unsigned(nblk), kThreads, 0, st>>>(nuniq, nseg, sc.bsum, uoff);
        count_total_kernel<<<1, 1, 0, st>>>(nuniq, uoff, nseg, total);
        kernels += 6;
    } else {
        count_light_kernel<true><<<gw, kThreads, 0, st>>>(sc.real, nseg, seglen, sc.counts, sc.offsets, nuniq, uoff,
                                                          sc.coltab, b, words, hits);
        count_heavy_kernel<true><<<gh, kThreads, 0, st>>>(sc.real, seglen, sc.counts, sc.offsets, sc.heavy_list,
                                                          sc.heavy_count, nuniq, uoff, sc.coltab, b, words, hits);
        kernels += 2;
    }
    return cudaGetLastError();
}

// One layout routine serves both the size query and the carving, so the two can
// never disagree.
static size_t layout(SamplerScratch *sc, uint8_t *base, uint64_t nseg, uint64_t shots, bool with_parts)
{
    const uint64_t nblk = (nseg + kScanBlock - 1) / kScanBlock;
    size_t b = 0;
    auto take = [&](size_t x) {
        uint8_t *p = base ? base + b : nullptr;
        b += (x + 255) & ~size_t(255);
        return p;
    };
    uint8_t *segcdf = take(nseg * 8);
    uint8_t *fb = base ? base + b : nullptr;
    uint8_t *heavy_count = take(16);
    uint8_t *fe = base ? base + b : nullptr;
    uint8_t *counts = take(nseg * 8);
    uint8_t *offsets = take(nseg * 8);
    uint8_t *bsum = take(nblk * 8);
    uint8_t *heavy = take(nseg * 4);
    uint8_t *real = take(shots * 8);
    uint8_t *words = take(shots * 8);
    uint8_t *coltab = take(8 * 256 * 8);
    uint8_t *parts = with_parts ? take(nseg * 32 * 8) : nullptr;
    if (sc) {
        sc->parts = reinterpret_cast<double *>(parts);
        sc->segcdf = reinterpret_cast<double *>(segcdf);
        sc->flags_begin = fb;
        sc->heavy_count = reinterpret_cast<uint32_t *>(heavy_count);
        sc->flags_end = fe;
        sc->counts = reinterpret_cast<unsigned long long *>(counts);
        sc->offsets = reinterpret_cast<unsigned long long *>(offsets);
        sc->bsum = reinterpret_cast<unsigned long long *>(bsum);
        sc->heavy_list = reinterpret_cast<uint32_t *>(heavy);
        sc->real = reinterpret_cast<uint64_t *>(real);
        sc->words = reinterpret_cast<uint64_t *>(words);
        sc->coltab = reinterpret_cast<uint64_t *>(coltab);
    }
    return b;
}

size_t SamplerScratch::need_bytes(uint64_t nseg, uint64_t shots, bool parts)
{
    return layout(nullptr, nullptr, nseg, shots, parts);
}

void SamplerScratch::carve(uint8_t *base, uint64_t nseg, uint64_t shots, bool parts)
{
    layout(this, base, nseg, shots, parts);
}

cudaError_t run_sampler(const void *state, int elem_bytes, int m, uint64_t shots, uint64_t stream_seed,
                        const uint64_t *host_coltab, uint64_t b, SamplerScratch &sc, DevStatus *status, int sms,
                        cudaStream_t st, uint64_t &kernels)
{
    const uint64_t local = 1ULL << m;
    const uint32_t seglen = uint32_t(std::min<uint64_t>(4096, local));
    const uint64_t nseg = local / seglen;
    const uint64_t nblk = (nseg + kScanBlock - 1) / kScanBlock;
    const uint64_t stream2 = mix_seed_host(stream_seed, 1);
    cudaError_t e;
    e = cudaMemsetAsync(sc.flags_begin, 0, size_t(static_cast<uint8_t *>(sc.flags_end) - static_cast<uint8_t *>(sc.flags_begin)), st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(sc.counts, 0, nseg * 8, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(sc.coltab, host_coltab, 8 * 256 * 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const unsigned gmass = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((nseg * 32 + kThreads - 1) / kThreads,
                                                                             uint64_t(sms) * 8)));
    if (elem_bytes == 8)
        seg_mass_kernel<float2><<<gmass, kThreads, 0, st>>>(static_cast<const float2 *>(state), nseg, seglen, sc.segcdf,
                                                            sc.parts);
    else
        seg_mass_kernel<double2><<<gmass, kThreads, 0, st>>>(static_cast<const double2 *>(state), nseg, seglen,
                                                            sc.segcdf, sc.parts);
    double *bsum_d = reinterpret_cast<double *>(sc.bsum);  // the counts' scan reuses it afterwards
    block_sum_kernel<double><<<unsigned(nblk), kThreads, 0, st>>>(sc.segcdf, nseg, bsum_d);
    scan_small_kernel<double><<<1, 32, 0, st>>>(bsum_d, nblk);
    block_scan_kernel<double, true><<<unsigned(nblk), kThreads, 0, st>>>(sc.segcdf, nseg, bsum_d, sc.segcdf);
    const unsigned gc = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((shots + kThreads - 1) / kThreads, uint64_t(sms) * 8)));
    count_kernel<<<gc, kThreads, 0, st>>>(sc.segcdf, nseg, stream_seed, shots, sc.counts);
    block_sum_kernel<unsigned long long><<<unsigned(nblk), kThreads, 0, st>>>(sc.counts, nseg, sc.bsum);
    scan_small_kernel<unsigned long long><<<1, 32, 0, st>>>(sc.bsum, nblk);
    block_scan_kernel<unsigned long long, false><<<unsigned(nblk), kThreads, 0, st>>>(sc.counts, nseg, sc.bsum,
                                                                                     sc.offsets);
    const uint64_t warps_needed = (nseg + 31) / 32;
    const unsigned gw = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((warps_needed * 32 + kThreads - 1) / kThreads,
                                                                          uint64_t(sms) * 8)));
    if (elem_bytes == 8)
        resolve_warp_kernel<float2><<<gw, kThreads, 0, st>>>(static_cast<const float2 *>(state), nseg, seglen, sc.counts,
                                                            sc.offsets, stream2, sc.real, sc.heavy_list, sc.heavy_count,
                                                            sc.parts);
    else
        resolve_warp_kernel<double2><<<gw, kThreads, 0, st>>>(static_cast<const double2 *>(state), nseg, seglen,
                                                             sc.counts, sc.offsets, stream2, sc.real, sc.heavy_list,
                                                             sc.heavy_count, sc.parts);
    const size_t smem = size_t(seglen + seglen / 16 + 1) * 8;
    const unsigned gh = unsigned(sms) * 2;
    if (elem_bytes == 8)
        resolve_cta_kernel<float2><<<gh, kThreads, smem, st>>>(static_cast<const float2 *>(state), seglen, sc.counts,
                                                              sc.offsets, stream2, sc.real, sc.heavy_list,
                                                              sc.heavy_count);
    else
        resolve_cta_kernel<double2><<<gh, kThreads, smem, st>>>(static_cast<const double2 *>(state), seglen, sc.counts,
                                                               sc.offsets, stream2, sc.real, sc.heavy_list,
                                                               sc.heavy_count);
    const unsigned gm = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((shots + kThreads - 1) / kThreads, uint64_t(sms) * 8)));
    map_kernel<<<gm, kThreads, 0, st>>>(sc.real, shots, sc.coltab, b, sc.words);
    kernels += 11;
    (void)status;  // no step of the draw waits on another CTA
    return cudaGetLastError();
}

// The same draw as run_sampler up to the real indices, written to a caller buffer;
// used by the allocation-free entry point (noalloc.cu). Scratch comes from sc,
// whose flag region, counts and heavy count the caller has cleared.
cudaError_t run_sampler_real(const void *state, int elem_bytes, int m, uint64_t shots, uint64_t stream_seed,
                             uint64_t *real_out, SamplerScratch &sc, DevStatus *status, int sms, cudaStream_t st)
{
    const uint64_t local = 1ULL << m;
    const uint32_t seglen = uint32_t(std::min<uint64_t>(4096, local));
    const uint64_t nseg = local / seglen;
    const uint64_t nblk = (nseg + kScanBlock - 1) / kScanBlock;
    const uint64_t stream2 = mix_seed_host(stream_seed, 1);
    const unsigned gmass = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((nseg * 32 + kThreads - 1) / kThreads,
                                                                             uint64_t(sms) * 8)));
    if (elem_bytes == 8)
        seg_mass_kernel<float2><<<gmass, kThreads, 0, st>>>(static_cast<const float2 *>(state), nseg, seglen, sc.segcdf,
                                                            sc.parts);
    else
        seg_mass_kernel<double2><<<gmass, kThreads, 0, st>>>(static_cast<const double2 *>(state), nseg, seglen,
                                                            sc.segcdf, sc.parts);
    double *bsum_d = reinterpret_cast<double *>(sc.bsum);  // the counts' scan reuses it afterwards
    block_sum_kernel<double><<<unsigned(nblk), kThreads, 0, st>>>(sc.segcdf, nseg, bsum_d);
    scan_small_kernel<double><<<1, 32, 0, st>>>(bsum_d, nblk);
    block_scan_kernel<double, true><<<unsigned(nblk), kThreads, 0, st>>>(sc.segcdf, nseg, bsum_d, sc.segcdf);
    const unsigned gc = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((shots + kThreads - 1) / kThreads, uint64_t(sms) * 8)));
    count_kernel<<<gc, kThreads, 0, st>>>(sc.segcdf, nseg, stream_seed, shots, sc.counts);
    block_sum_kernel<unsigned long long><<<unsigned(nblk), kThreads, 0, st>>>(sc.counts, nseg, sc.bsum);
    scan_small_kernel<unsigned long long><<<1, 32, 0, st>>>(sc.bsum, nblk);
    block_scan_kernel<unsigned long long, false><<<unsigned(nblk), kThreads, 0, st>>>(sc.counts, nseg, sc.bsum,
                                                                                     sc.offsets);
    const uint64_t warps_needed = (nseg + 31) / 32;
    const unsigned gw = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((warps_needed * 32 + kThreads - 1) / kThreads,
                                                                          uint64_t(sms) * 8)));
    if (elem_bytes == 8)
        resolve_warp_kernel<float2><<<gw, kThreads, 0, st>>>(static_cast<const float2 *>(state), nseg, seglen, sc.counts,
                                                            sc.offsets, stream2, real_out, sc.heavy_list, sc.heavy_count,
                                                            sc.parts);
    else
        resolve_warp_kernel<double2><<<gw, kThreads, 0, st>>>(static_cast<const double2 *>(state), nseg, seglen,
                                                             sc.counts, sc.offsets, stream2, real_out, sc.heavy_list,
                                                             sc.heavy_count, sc.parts);
    const size_t smem = size_t(seglen + seglen / 16 + 1) * 8;
    const unsigned gh = unsigned(sms) * 2;
    if (elem_bytes == 8)
        resolve_cta_kernel<float2><<<gh, kThreads, smem, st>>>(static_cast<const float2 *>(state), seglen, sc.counts,
                                                              sc.offsets, stream2, real_out, sc.heavy_list,
                                                              sc.heavy_count);
    else
        resolve_cta_kernel<double2><<<gh, kThreads, smem, st>>>(static_cast<const double2 *>(state), seglen, sc.counts,
                                                               sc.offsets, stream2, real_out, sc.heavy_list,
                                                               sc.heavy_count);
    (void)status;  // no step of the draw waits on another CTA
    return cudaGetLastError();
}

uint64_t mix_seed_host(uint64_t base, uint64_t salt)
{
    // mix_seed, measure_cuda.cu:103-109
    uint64_t z = base + 0x9e3779b97f4a7c15ULL + salt;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

}  // namespace zxh
