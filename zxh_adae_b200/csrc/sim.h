// sim.h -- the zxh_sim handle behind the extern "C" boundary and the helpers the
// boundary's translation units share (capi.cpp, adjoint_api.cpp).
#pragma once

#include "../../include/zxh_b200.h"
#include "host.h"
#include "sampler.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

using zxh::Gate;

struct zxh_sim {
    size_t n = 0;
    bool disable_x = false, eager = false;
    int dtype = ZXH_C128, elem_bytes = 16, device = 0, sms = 148;
    std::vector<Gate> gates;
    bool use_seed = false;
    uint64_t seed = 0;
    std::string err;
    cudaStream_t stream = nullptr;

    void *d_state = nullptr;
    size_t state_cap_bytes = 0;
    int M = 0;
    zxh::WalkState ws;
    bool executed = false;
    // phases due on the state that the last zxh_apply / zxh_apply_async left over
    // (the real split's P(b) and global phase after its last U3 batch): the next
    // apply takes them into its first window; every call that reads the state
    // applies them first (flush_pending)
    std::vector<zxh::DiagTerm> pending;

    uint8_t *d_blob = nullptr;
    size_t blob_cap = 0;
    uint8_t *h_stage = nullptr;
    size_t stage_cap = 0;
    zxh::DevStatus *d_status = nullptr;
    zxh::DevStatus *h_status = nullptr;

    uint8_t *d_samp = nullptr;
    size_t samp_cap = 0;
    zxh::SamplerScratch sc;
    size_t measured = 0;
    int measured_m = 0;  // log2 amplitudes of the state the last draw read

    // counts of the last draw (zxh_counts): per-segment distinct outcomes and
    // their scan, the total, then the (word, count) pairs
    uint8_t *d_cnt = nullptr;
    size_t cnt_cap = 0;
    bool cnt_ready = false;  // pass 1 ran for the current draw
    uint64_t cnt_total = 0;

    void *d_out = nullptr;
    size_t out_cap = 0;

    // zxh_apply_async: two pinned program slots (each reused once the upload that
    // last read it has run, an event per slot) and whether work is in flight
    uint8_t *h_async[2] = {nullptr, nullptr};
    size_t async_cap = 0;
    cudaEvent_t async_ev[2] = {nullptr, nullptr};
    int async_slot = 0;
    bool async_pending = false;

    uint64_t stat_kernels = 0, stat_passes = 0;
    float last_ms = 0.0f;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evf0 = nullptr, evf1 = nullptr;  // the adjoint sweep's forward part
    zxh::PlanParams pp;

    // adjoint sweep: the reverse copy of the state, lambda, forward checkpoints,
    // and a small region for terms, diagonal groups, gradients and the energy
    void *d_psi = nullptr, *d_lam = nullptr, *d_ckpt = nullptr;
    size_t psi_cap = 0, lam_cap = 0, ckpt_cap = 0;
    uint8_t *d_adj = nullptr;
    size_t adj_cap = 0;
};

namespace zxh {
namespace api {

constexpr double kPi = 3.14159265358979323846;

// Records msg as the handle's (or the thread's, for a null handle) last error.
int fail(zxh_sim *s, int code, const std::string &msg);
int cuda_fail(zxh_sim *s, cudaError_t e, const char *what);
// Makes the handle's device current and settles zxh_apply_async work in flight
// (waits for it and returns the error a step recorded, if any).
int use_device(zxh_sim *s);
// Grows a device allocation to at least need bytes (contents are not kept).
int ensure_dev(zxh_sim *s, void **p, size_t &cap, size_t need, const char *what);
// Lowers one record the way the reference's recorders do (zxh.cpp:234-310).
int lower(zxh_sim *s, const zxh_gate &g, std::vector<Gate> &out);
// Uploads the plan, runs it on the handle's stream and waits for the device.
int run_plan(zxh_sim *s, const zxh::Plan &pl);
// Applies the phases a previous apply left over (sim.pending), if any: one
// diagonal pass, run like a plan (its device time in the handle's stats).
int flush_pending(zxh_sim *s);

}  // namespace api
}  // namespace zxh

#define CK(s, call, what)                                                   \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) return zxh::api::cuda_fail(s, e_, what);     \
    } while (0)
