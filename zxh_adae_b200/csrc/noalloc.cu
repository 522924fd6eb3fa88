// noalloc.cu -- the multinomial sampler for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc: a serving process that
// reserves all of its device memory once at start-up and must never grow it
// afterwards, a framework whose own caching allocator owns the device and forbids
// raw allocations next to it, and host threads on a latency-critical path that
// must not take the CUDA allocator's locks or pay its first-touch costs.
// zxh_sample_noalloc gives them the sampler of zxh_measure with no allocation at
// all: the caller owns the state (a device pointer) and the output buffer (a
// device pointer), and every piece of working memory lives in one file-scope
// __device__ array below.
//
// Limits and sharing rules:
//  * the array holds the scratch of states up to 2^28 amplitudes (2^16 segments
//    of 2^12); larger states are rejected with ZXH_ERR_LIMIT before any work;
//  * every GPU that loads this library keeps the array (2.25 MiB) until exit;
//  * all calls on a device share the one array, so calls that overlap on the
//    GPU (different streams, or threads racing) corrupt each other's draws;
//    serialise them. Each call clears the parts that must start at zero;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current) and keeps
//    it for the life of the process; make that first call before any stream
//    capture begins. The kept address belongs to the device's primary context:
//    after cudaDeviceReset the process must not call this entry point again.
#include "../../include/zxh_b200.h"
#include "core.h"
#include "sampler.h"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace zxh {
void set_thread_error(const std::string &msg);  // capi.cpp: message for zxh_last_error(NULL)
}

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(2304) << 10;  // 2.25 MiB
constexpr int kMaxBits = 28;                                 // 2^28 amplitudes, 2^16 segments
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host-side view: device address of g_noalloc_scratch and SM count, per device.
void *g_scratch_ptr[kMaxDevices] = {nullptr};
int g_scratch_sms[kMaxDevices] = {0};
std::mutex g_setup_mutex;

int fail(int code, const std::string &msg)
{
    zxh::set_thread_error(msg);
    return code;
}

}  // namespace

extern "C" int zxh_sample_noalloc(const void *state, int dtype, size_t m_bits, uint64_t seed, size_t shots,
                                  uint64_t *real_out, void *stream)
{
    if (!state) return fail(ZXH_ERR_ARG, "zxh_sample_noalloc: state is null");
    if (dtype != ZXH_C64 && dtype != ZXH_C128) return fail(ZXH_ERR_ARG, "zxh_sample_noalloc: dtype must be ZXH_C64 or ZXH_C128");
    if (m_bits > size_t(kMaxBits))
        return fail(ZXH_ERR_LIMIT, "zxh_sample_noalloc: state of 2^" + std::to_string(m_bits) +
                                       " amplitudes exceeds the static scratch limit of 2^28");
    if (shots == 0) return ZXH_OK;
    if (!real_out) return fail(ZXH_ERR_ARG, "zxh_sample_noalloc: real_out is null");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(ZXH_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(ZXH_ERR_LIMIT, "zxh_sample_noalloc: device ordinal too large");
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return fail(ZXH_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            int sms = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return fail(ZXH_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
            g_scratch_sms[dev] = sms;
            g_scratch_ptr[dev] = p;
        }
    }
    uint8_t *base = static_cast<uint8_t *>(g_scratch_ptr[dev]);
    const int m = int(m_bits);
    const uint64_t local = 1ULL << m;
    const uint64_t seglen = local < 4096 ? local : 4096;
    const uint64_t nseg = local / seglen;
    if (zxh::SamplerScratch::need_bytes(nseg, 0) > kNoAllocScratchBytes)
        return fail(ZXH_ERR_LIMIT, "zxh_sample_noalloc: scratch layout exceeds the static array");
    zxh::SamplerScratch sc;
    sc.carve(base, nseg, 0);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // the previous call's contents stay in the array: clear what starts at zero
    e = cudaMemsetAsync(sc.flags_begin, 0,
                        size_t(static_cast<uint8_t *>(sc.flags_end) - static_cast<uint8_t *>(sc.flags_begin)), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc.counts, 0, nseg * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail(ZXH_ERR_CUDA, std::string("clear scratch: ") + cudaGetErrorString(e));

    const uint64_t stream_seed = zxh::mix_seed_host(seed, 0);  // as zxh_measure with a set seed
    // no step of the draw waits on another CTA, so there is no device status to read back
    e = zxh::run_sampler_real(state, dtype == ZXH_C64 ? 8 : 16, m, shots, stream_seed, real_out, sc, nullptr,
                              g_scratch_sms[dev], st);
    if (e != cudaSuccess) return fail(ZXH_ERR_CUDA, std::string("sampler launch: ") + cudaGetErrorString(e));
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(ZXH_ERR_CUDA, std::string("sampler: ") + cudaGetErrorString(e));
    return ZXH_OK;
}
