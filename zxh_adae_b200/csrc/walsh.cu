// walsh.cu -- the diagonal window as a Walsh sum (sm_100a): one read-modify-write
// of the state for a window of commuting P / CP / RZ / Z gates whose selectors are
// parities of several real-address bits (what X / CX transport makes of them).
//
// The reference evaluates every such gate per amplitude with selector bit tests
// (src/zxh/src/kernel/kernel_cuda.cu:577-603). Here the window is first rewritten
// on the host: with [S] = (1 - (-1)^S) / 2 for a selector S = parity(alpha & r) ^ beta,
//   theta [S0]       = 2q - 2q s0 X(a0)
//   theta [S0] [S1]  = q - q s0 X(a0) - q s1 X(a1) + q s0 s1 X(a0 ^ a1)
// where q = theta / 4 (in turns), s = (-1)^beta and X(a) = (-1)^parity(a & r). Terms
// with the same mask merge, so a window is a constant plus one coefficient W(g) per
// distinct mask g, at most n + n(n-1)/2 of them however many gates it holds.
//
// On the device a warp owns tiles of 2^T contiguous amplitudes (T = 10 for
// complex64, 9 for complex128). Splitting a mask g into its in-tile part g_lo and
// out-of-tile part g_hi, the phase at in-tile offset e of tile t is
//   C + sum_{g_lo} U_t(g_lo) (-1)^parity(g_lo & e),  U_t(g_lo) = sum W(g) (-1)^parity(g_hi & t),
// i.e. C plus the Walsh-Hadamard transform of U_t. Per tile the warp builds U_t in
// its shared-memory slab (each lane sums a contiguous slice of the term list, which
// the host sorts by g_lo and the CTA stages in shared memory, and adds each run
// with one shared atomic), then transforms it in two halves: read with the
// register index on the bits that are lane bits of the amplitude layout (transform
// those in registers), written back, read again in the amplitude layout (transform
// the slot and row bits in registers). The slab is XOR-swizzled so both reads are
// free of bank conflicts; complex128 keeps one lane bit for a shuffle stage. The
// phase arithmetic is integer (32-bit turns for complex64, 64-bit for complex128),
// so every sum is exact modulo a turn; the complex64 coefficients are rounded once
// to 2^-32 turns. The cost per amplitude is fixed (T butterflies, one
// table-plus-Taylor exp, one complex multiply) whatever the window's size or the
// affine map.
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>
#include <type_traits>

namespace zxh {

namespace {

constexpr int kWalshRowBits = 4;       // register rows per lane: 16
constexpr uint32_t kWalshSmemTerms = 1024;  // terms staged in shared memory (more are read from global)

template <typename E>
struct WalshShape {
    static constexpr int V = ET<E>::V;             // amplitudes per 16-byte vector
    static constexpr int LV = V == 2 ? 1 : 0;      // vector-slot bit
    static constexpr int ROWS = 1 << kWalshRowBits;
    static constexpr int T = LV + 5 + kWalshRowBits;  // tile bits: 10 (complex64), 9 (complex128)
    using PT = typename std::conditional<V == 2, uint32_t, unsigned long long>::type;  // phase turns
};

__device__ __forceinline__ uint32_t to_phase(int64_t w, uint32_t *) { return turns32(w); }
__device__ __forceinline__ unsigned long long to_phase(int64_t w, unsigned long long *)
{
    return static_cast<unsigned long long>(w);
}

__device__ __forceinline__ float2 phase_mul(float2 a, uint32_t th, const float2 *tab)
{
    return cmul(a, phase_factor32(tab, th));
}
__device__ __forceinline__ double2 phase_mul(double2 a, unsigned long long th, const double2 *tab)
{
    return cmul(a, phase_factor(tab, static_cast<int64_t>(th)));
}

// Slab slot of in-tile index g. complex64 (T = 10, 4-byte slots): bits 1..4 XOR
// bits 6..9; complex128 (T = 9, 8-byte slots): bits 0..3 XOR bits 5..8. Either way
// the read with lanes on the amplitude layout's row bits and the read with lanes
// on its lane bits both spread over all banks.
template <int V>
__device__ __forceinline__ uint32_t wslot(uint32_t g)
{
    if constexpr (V == 2) return g ^ (((g >> 6) & 15u) << 1);
    else return g ^ ((g >> 5) & 15u);
}

// Butterflies over register index bits [0, NB) of a[]: (x, y) -> (x + y, x - y).
template <int NB, int N, typename PT>
__device__ __forceinline__ void wht_regs(PT (&a)[N])
{
#pragma unroll
    for (int r = 0; r < NB; r++)
#pragma unroll
        for (int j = 0; j < N; j++)
            if (!((j >> r) & 1)) {
                const PT x = a[j], y = a[j | (1 << r)];
                a[j] = x + y;
                a[j | (1 << r)] = x - y;
            }
}

template <typename E>
__global__ void __launch_bounds__(kThreads, 2) walsh_kernel(const uint8_t *__restrict__ blob, uint64_t woff,
                                                            uint64_t toff, E *__restrict__ state, uint64_t ntiles)
{
    using S = WalshShape<E>;
    using VT = typename ET<E>::VT;
    using PT = typename S::PT;
    constexpr int V = S::V, LV = S::LV, ROWS = S::ROWS, T = S::T;
    constexpr int WARPS = kThreads / 32;

    __shared__ E s_exp[1 << kExpTableBits];
    __shared__ __align__(16) PT s_u[WARPS][1 << T];
    extern __shared__ __align__(128) WalshTermDev s_terms[];  // min(n_terms, kWalshSmemTerms) staged terms

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const WalshDev &d = *reinterpret_cast<const WalshDev *>(blob + woff);
    const WalshTermDev *gterms = reinterpret_cast<const WalshTermDev *>(blob + d.off_terms);
    const E *tab = reinterpret_cast<const E *>(blob + toff);
    for (int i = tid; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = tab[i];
    for (int i = tid; i < WARPS * (1 << T); i += kThreads) (&s_u[0][0])[i] = 0;
    const bool staged = d.n_terms <= kWalshSmemTerms;  // the launch sized s_terms for this
    if (staged)
        for (uint32_t i = uint32_t(tid); i < d.n_terms; i += kThreads) s_terms[i] = gterms[i];
    __syncthreads();
    const WalshTermDev *terms = staged ? s_terms : gterms;

    const PT c0 = to_phase(d.c0, static_cast<PT *>(nullptr));
    // this lane's slice of the term list (sorted by g)
    const uint32_t per = (d.n_terms + 31u) / 32u;
    const uint32_t t_lo = min(d.n_terms, uint32_t(lane) * per), t_hi = min(d.n_terms, t_lo + per);
    PT *su = s_u[warp];
    constexpr uint64_t kHiMask = (1ULL << kWalshGShift) - 1ULL;

    const uint64_t stride = uint64_t(gridDim.x) * WARPS;
    constexpr uint32_t kTileBytes = uint32_t(sizeof(E)) << T;
    uint64_t tile = uint64_t(blockIdx.x) * WARPS + uint64_t(warp);
    if (lane == 0 && tile < ntiles) bulk_prefetch_l2(state + (tile << T), kTileBytes);
    for (; tile < ntiles; tile += stride) {
        E *base = state + (tile << T);
        // 1. the warp's next tile is fetched into L2 while this one is worked on
        if (lane == 0 && tile + stride < ntiles) bulk_prefetch_l2(state + ((tile + stride) << T), kTileBytes);

        // 2. U_t in the slab: runs of equal g summed per lane, one atomic each
        uint32_t gcur = 0xffffffffu;
        PT acc = 0;
        for (uint32_t i = t_lo; i < t_hi; i++) {
            const WalshTermDev tm = terms[i];
            PT w = to_phase(tm.w, static_cast<PT *>(nullptr));
            if (par64(tm.hi_g & kHiMask & tile)) w = PT(0) - w;
            const uint32_t g = uint32_t(tm.hi_g >> kWalshGShift);
            if (g != gcur) {
                if (gcur != 0xffffffffu) atomicAdd(&su[wslot<V>(gcur)], acc);
                gcur = g;
                acc = 0;
            }
            acc += w;
        }
        if (gcur != 0xffffffffu) atomicAdd(&su[wslot<V>(gcur)], acc);
        __syncwarp();

        // 3. first half of the transform: registers on the bits that are lane bits
        //    of the amplitude layout (complex64: e1..e5, lanes on e0, e6..e9;
        //    complex128: e0..e3, lanes on e4..e8)
        PT u[ROWS][V];
        {
            constexpr int NY = V == 2 ? 32 : 16;
            PT y[NY];
            auto gy = [&](int r) -> uint32_t {
                if constexpr (V == 2) return uint32_t(lane & 1) | (uint32_t(r) << 1) | (uint32_t(lane >> 1) << 6);
                else return uint32_t(r) | (uint32_t(lane & 1) << 4) | (uint32_t(lane >> 1) << 5);
            };
#pragma unroll
            for (int r = 0; r < NY; r++) y[r] = su[wslot<V>(gy(r))];
            wht_regs<V == 2 ? 5 : 4>(y);
#pragma unroll
            for (int r = 0; r < NY; r++) su[wslot<V>(gy(r))] = y[r];
        }
        __syncwarp();
        // 4. the tile's rows (all in flight at once; L2 has them or is fetching them),
        //    then the second half of the transform in the amplitude layout (slot bit
        //    and row bits in registers; complex128's lane bit 4 by shuffles); the
        //    slab is cleared behind the read
        VT x[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; j++)
            x[j] = __ldcs(reinterpret_cast<const VT *>(base + ((uint32_t(j) << (LV + 5)) | (uint32_t(lane) << LV))));
#pragma unroll
        for (int j = 0; j < ROWS; j++) {
            const uint32_t e0 = (uint32_t(j) << (LV + 5)) | (uint32_t(lane) << LV);
            if constexpr (V == 2) {
                uint2 *pp = reinterpret_cast<uint2 *>(&su[wslot<V>(e0)]);
                const uint2 pv = *pp;
                u[j][0] = pv.x + pv.y;
                u[j][1] = pv.x - pv.y;
                *pp = make_uint2(0u, 0u);
            } else {
                PT *pp = &su[wslot<V>(e0)];
                u[j][0] = *pp;
                *pp = 0;
            }
        }
        if constexpr (V == 1) {
            const bool up = (lane >> 4) & 1;
#pragma unroll
            for (int j = 0; j < ROWS; j++) {
                const PT o = __shfl_xor_sync(0xffffffffu, u[j][0], 16);
                u[j][0] = up ? o - u[j][0] : u[j][0] + o;
            }
        }
#pragma unroll
        for (int r = 0; r < kWalshRowBits; r++)
#pragma unroll
            for (int j = 0; j < ROWS; j++)
                if (!((j >> r) & 1)) {
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        const PT a = u[j][v], b = u[j | (1 << r)][v];
                        u[j][v] = a + b;
                        u[j | (1 << r)][v] = a - b;
                    }
                }
        __syncwarp();

        // 5. phases applied, rows written back
#pragma unroll
        for (int j = 0; j < ROWS; j++) {
            VT o = x[j];
#pragma unroll
            for (int v = 0; v < V; v++) vset(o, v, phase_mul(vget(o, v), c0 + u[j][v], s_exp));
            __stcs(reinterpret_cast<VT *>(base + ((uint32_t(j) << (LV + 5)) | (uint32_t(lane) << LV))), o);
        }
    }
}

template <typename E>
cudaError_t launch_walsh(const uint8_t *dblob, uint64_t woff, uint64_t toff, int m, uint32_t n_terms, E *state,
                         int sms, cudaStream_t st)
{
    constexpr int T = WalshShape<E>::T;
    if (m < T) return cudaErrorInvalidValue;
    const uint64_t ntiles = 1ULL << (m - T);
    // the term list is staged in dynamic shared memory when it has at most
    // kWalshSmemTerms entries (the count is in the device blob: the host passes the
    // size it compiled)
    const size_t smem = size_t(n_terms <= kWalshSmemTerms ? n_terms : 0) * sizeof(WalshTermDev);
    cudaError_t e = cudaFuncSetAttribute(walsh_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(kWalshSmemTerms * sizeof(WalshTermDev)));
    if (e != cudaSuccess) return e;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, walsh_kernel<E>, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const uint64_t warps = ntiles;
    const uint64_t ctas = (warps + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ctas, uint64_t(sms) * uint64_t(per_sm))));
    walsh_kernel<E><<<grid, kThreads, smem, st>>>(dblob, woff, toff, state, ntiles);
    return cudaGetLastError();
}

}  // namespace

int walsh_tile_bits(int elem_bytes) { return elem_bytes == 8 ? WalshShape<float2>::T : WalshShape<double2>::T; }

cudaError_t run_walsh(const uint8_t *dblob, uint64_t woff, uint64_t toff, int m, uint32_t n_terms, int elem_bytes,
                      void *state, int sms, cudaStream_t st)
{
    if (elem_bytes == 8)
        return launch_walsh<float2>(dblob, woff, toff, m, n_terms, static_cast<float2 *>(state), sms, st);
    return launch_walsh<double2>(dblob, woff, toff, m, n_terms, static_cast<double2 *>(state), sms, st);
}

}  // namespace zxh
