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
// shared memory (each lane sums a contiguous slice of the term list, which the host
// sorts by g_lo, and adds each run with one shared atomic), loads it into registers
// in the layout of its amplitudes (bit 0: vector slot, bits 1..5: lane, upper bits:
// register rows; complex128 has no slot bit), and transforms it: slot and row bits
// in registers, lane bits with shuffles. The phase arithmetic is integer (32-bit
// turns for complex64, 64-bit for complex128), so every sum is exact modulo a turn;
// the complex64 coefficients are rounded once to 2^-32 turns. The cost per
// amplitude is fixed (T butterflies, one table-plus-Taylor exp, one complex
// multiply) whatever the window's size or the affine map.
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>
#include <type_traits>

namespace zxh {

namespace {

constexpr int kWalshRowBits = 4;  // register rows per lane: 16

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

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const E *tab = reinterpret_cast<const E *>(blob + toff);
    for (int i = tid; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = tab[i];
    for (int i = tid; i < WARPS * (1 << T); i += kThreads) (&s_u[0][0])[i] = 0;
    __syncthreads();

    const WalshDev &d = *reinterpret_cast<const WalshDev *>(blob + woff);
    const WalshTermDev *terms = reinterpret_cast<const WalshTermDev *>(blob + d.off_terms);
    const PT c0 = to_phase(d.c0, static_cast<PT *>(nullptr));
    // this lane's slice of the term list (sorted by g_lo)
    const uint32_t per = (d.n_terms + 31u) / 32u;
    const uint32_t t_lo = min(d.n_terms, uint32_t(lane) * per), t_hi = min(d.n_terms, t_lo + per);
    PT *su = s_u[warp];

    const uint64_t stride = uint64_t(gridDim.x) * WARPS;
    for (uint64_t tile = uint64_t(blockIdx.x) * WARPS + uint64_t(warp); tile < ntiles; tile += stride) {
        E *base = state + (tile << T);
        // 1. every row of the tile in flight before any arithmetic
        VT x[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; j++)
            x[j] = __ldcs(reinterpret_cast<const VT *>(base + ((uint32_t(j) << (LV + 5)) | (uint32_t(lane) << LV))));

        // 2. U_t in shared memory: runs of equal g_lo summed per lane, one atomic each
        uint32_t gcur = 0xffffffffu;
        PT acc = 0;
        for (uint32_t i = t_lo; i < t_hi; i++) {
            const WalshTermDev tm = terms[i];
            PT w = to_phase(tm.w, static_cast<PT *>(nullptr));
            if (par64(tm.hi & tile)) w = PT(0) - w;
            if (tm.g != gcur) {
                if (gcur != 0xffffffffu) atomicAdd(&su[gcur], acc);
                gcur = tm.g;
                acc = 0;
            }
            acc += w;
        }
        if (gcur != 0xffffffffu) atomicAdd(&su[gcur], acc);
        __syncwarp();

        // 3. U_t into registers in the amplitudes' layout, then cleared for the next tile
        PT u[ROWS][V];
#pragma unroll
        for (int j = 0; j < ROWS; j++) {
            const uint32_t e0 = (uint32_t(j) << (LV + 5)) | (uint32_t(lane) << LV);
            if constexpr (V == 2) {
                const uint2 p = *reinterpret_cast<const uint2 *>(&su[e0]);
                u[j][0] = p.x;
                u[j][1] = p.y;
                *reinterpret_cast<uint2 *>(&su[e0]) = make_uint2(0u, 0u);
            } else {
                u[j][0] = su[e0];
                su[e0] = 0;
            }
        }
        __syncwarp();

        // 4. Walsh-Hadamard transform: slot bit, lane bits (shuffles), row bits
        if constexpr (V == 2) {
#pragma unroll
            for (int j = 0; j < ROWS; j++) {
                const PT a = u[j][0], b = u[j][1];
                u[j][0] = a + b;
                u[j][1] = a - b;
            }
        }
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const bool up = (lane >> k) & 1;
#pragma unroll
            for (int j = 0; j < ROWS; j++)
#pragma unroll
                for (int v = 0; v < V; v++) {
                    const PT y = __shfl_xor_sync(0xffffffffu, u[j][v], 1 << k);
                    u[j][v] = up ? y - u[j][v] : u[j][v] + y;
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

        // 5. phases applied, rows written back
#pragma unroll
        for (int j = 0; j < ROWS; j++) {
            VT y = x[j];
#pragma unroll
            for (int v = 0; v < V; v++) vset(y, v, phase_mul(vget(y, v), c0 + u[j][v], s_exp));
            __stcs(reinterpret_cast<VT *>(base + ((uint32_t(j) << (LV + 5)) | (uint32_t(lane) << LV))), y);
        }
    }
}

template <typename E>
cudaError_t launch_walsh(const uint8_t *dblob, uint64_t woff, uint64_t toff, int m, E *state, int sms,
                         cudaStream_t st)
{
    constexpr int T = WalshShape<E>::T;
    if (m < T) return cudaErrorInvalidValue;
    const uint64_t ntiles = 1ULL << (m - T);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, walsh_kernel<E>, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    const uint64_t warps = ntiles;
    const uint64_t ctas = (warps + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ctas, uint64_t(sms) * uint64_t(per_sm))));
    walsh_kernel<E><<<grid, kThreads, 0, st>>>(dblob, woff, toff, state, ntiles);
    return cudaGetLastError();
}

}  // namespace

int walsh_tile_bits(int elem_bytes) { return elem_bytes == 8 ? WalshShape<float2>::T : WalshShape<double2>::T; }

cudaError_t run_walsh(const uint8_t *dblob, uint64_t woff, uint64_t toff, int m, int elem_bytes, void *state, int sms,
                      cudaStream_t st)
{
    if (elem_bytes == 8) return launch_walsh<float2>(dblob, woff, toff, m, static_cast<float2 *>(state), sms, st);
    return launch_walsh<double2>(dblob, woff, toff, m, static_cast<double2 *>(state), sms, st);
}

}  // namespace zxh
