// capi.cpp -- the extern "C" boundary (include/zxh_b200.h) over the host core and
// the sm_100a kernels. One zxh_sim handle owns its gate list, device state, CUDA
// stream and scratch; handles are independent (the reference keeps its diagonal
// buckets and U3 descriptors in process-global statics, kernel_cuda.cu:91-142).
#include "../../include/zxh_b200.h"
#include "sim.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

using zxh::Gate;


namespace {
thread_local std::string g_create_error;
}  // namespace

namespace zxh {
namespace api {

int fail(zxh_sim *s, int code, const std::string &msg)
{
    if (s) s->err = msg;
    else g_create_error = msg;
    return code;
}

int cuda_fail(zxh_sim *s, cudaError_t e, const char *what)
{
    return fail(s, e == cudaErrorMemoryAllocation ? ZXH_ERR_OOM : ZXH_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

int use_device(zxh_sim *s)
{
    CK(s, cudaSetDevice(s->device), "cudaSetDevice");
    return zxh_sync(s);
}

int ensure_dev(zxh_sim *s, void **p, size_t &cap, size_t need, const char *what)
{
    if (need <= cap && *p) return ZXH_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    CK(s, cudaMalloc(p, need), what);
    cap = need;
    return ZXH_OK;
}

int check_q(zxh_sim *s, size_t q, const char *gate)
{
    if (q >= s->n) return fail(s, ZXH_ERR_ARG, std::string(gate) + " target qubit out of range");
    return ZXH_OK;
}

int push(zxh_sim *s, uint32_t t, size_t cq, size_t q, double th, double la, double ph)
{
    Gate g;
    g.type = t;
    g.cq = uint32_t(cq);
    g.q = uint32_t(q);
    g.reserved = 0;
    g.theta = th;
    g.lambda = la;
    g.phi = ph;
    s->gates.push_back(g);
    return ZXH_OK;
}


// Lowers one record the way the reference's recorders do (zxh.cpp:234-310).
int lower(zxh_sim *s, const zxh_gate &g, std::vector<Gate> &out)
{
    auto add = [&](uint32_t t, size_t cq, size_t q, double th, double la, double ph) {
        Gate r;
        r.type = t;
        r.cq = uint32_t(cq);
        r.q = uint32_t(q);
        r.reserved = 0;
        r.theta = th;
        r.lambda = la;
        r.phi = ph;
        out.push_back(r);
    };
    const bool two = g.type == ZXH_GATE_CRZ || g.type == ZXH_GATE_CP || g.type == ZXH_GATE_CX;
    if (g.type != ZXH_GATE_BARRIER && g.q >= s->n) return fail(s, ZXH_ERR_ARG, "gate target qubit out of range");
    if (two && g.cq >= s->n) return fail(s, ZXH_ERR_ARG, "gate control qubit out of range");
    switch (g.type) {
    case ZXH_GATE_BARRIER: add(zxh::G_BARRIER, 0, 0, 0, 0, 0); break;
    case ZXH_GATE_Z: add(zxh::G_Z, 0, g.q, 0, 0, 0); break;
    case ZXH_GATE_RZ: add(zxh::G_RZ, 0, g.q, g.theta, 0, 0); break;
    case ZXH_GATE_P: add(zxh::G_P, 0, g.q, g.theta, 0, 0); break;
    case ZXH_GATE_CRZ:
        add(zxh::G_P, 0, g.cq, -0.5 * g.theta, 0, 0);
        add(zxh::G_CP, g.cq, g.q, g.theta, 0, 0);
        break;
    case ZXH_GATE_CP: add(zxh::G_CP, g.cq, g.q, g.theta, 0, 0); break;
    case ZXH_GATE_X: add(zxh::G_X, 0, g.q, 0, 0, 0); break;
    case ZXH_GATE_CX: add(zxh::G_CX, g.cq, g.q, 0, 0, 0); break;
    case ZXH_GATE_H: add(zxh::G_H, 0, g.q, 0, 0, 0); break;
    case ZXH_GATE_U3: add(zxh::G_U3, 0, g.q, g.theta, g.lambda, g.phi); break;
    case ZXH_GATE_RX: add(zxh::G_U3, 0, g.q, g.theta, kPi / 2.0, -kPi / 2.0); break;
    default: return fail(s, ZXH_ERR_ARG, "unknown gate type " + std::to_string(g.type));
    }
    return ZXH_OK;
}

// Uploads the plan, runs it and waits for the device.
int run_plan(zxh_sim *s, const zxh::Plan &pl)
{
    const size_t bytes = std::max<size_t>(pl.blob.size(), 16);
    if (bytes > s->stage_cap) {
        if (s->h_stage) cudaFreeHost(s->h_stage);
        s->h_stage = nullptr;
        s->stage_cap = 0;
        CK(s, cudaMallocHost(reinterpret_cast<void **>(&s->h_stage), bytes * 2), "cudaMallocHost(program)");
        s->stage_cap = bytes * 2;
    }
    int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_blob), s->blob_cap, s->stage_cap, "cudaMalloc(program)");
    if (rc) return rc;
    std::memcpy(s->h_stage, pl.blob.data(), pl.blob.size());
    CK(s, cudaMemcpyAsync(s->d_blob, s->h_stage, pl.blob.size(), cudaMemcpyHostToDevice, s->stream), "upload program");
    CK(s, cudaMemsetAsync(s->d_status, 0, sizeof(zxh::DevStatus), s->stream), "reset status");
    uint64_t kernels = 0;
    CK(s, cudaEventRecord(s->ev0, s->stream), "event");
    CK(s, zxh::run_passes(pl.passes, s->d_blob, s->d_state, s->elem_bytes, s->d_status, s->sms, s->stream, kernels),
       "launch");
    CK(s, cudaEventRecord(s->ev1, s->stream), "event");
    CK(s, cudaMemcpyAsync(s->h_status, s->d_status, sizeof(zxh::DevStatus), cudaMemcpyDeviceToHost, s->stream),
       "read status");
    CK(s, cudaStreamSynchronize(s->stream), "execute");
    CK(s, cudaEventElapsedTime(&s->last_ms, s->ev0, s->ev1), "event time");
    s->stat_kernels = kernels;
    s->stat_passes = 0;
    for (const zxh::Pass &p : pl.passes)
        if (p.kind != zxh::Pass::PRODUCT) s->stat_passes++;
    if (s->h_status->code != 0)
        return fail(s, int(s->h_status->code),
                    "device wait gave up (site " + std::to_string(s->h_status->where) + ")");
    return ZXH_OK;
}

int flush_pending(zxh_sim *s)
{
    if (s->pending.empty()) return ZXH_OK;
    zxh::Plan pl;
    std::string err;
    if (int rc = zxh::plan(std::vector<zxh::Op>(), s->elem_bytes, s->pp, s->ws, pl, err, &s->pending, nullptr))
        return fail(s, rc, err);
    if (int rc = run_plan(s, pl)) return rc;
    s->pending.clear();
    return ZXH_OK;
}

void column_tables(const zxh::AffineMap &A, uint64_t tab[8][256])
{
    uint64_t col[64] = {0};
    for (int q = 0; q < A.n(); q++)
        for (int c = 0; c < A.m(); c++)
            if ((A.row(q) >> c) & 1) col[c] |= 1ULL << q;
    for (int k = 0; k < 8; k++)
        for (int byte = 0; byte < 256; byte++) {
            uint64_t v = 0;
            for (int i = 0; i < 8; i++)
                if ((byte >> i) & 1) v ^= col[8 * k + i];
            tab[k][byte] = v;
        }
}

}  // namespace api

void set_thread_error(const std::string &msg) { g_create_error = msg; }
}  // namespace zxh

using namespace zxh::api;

extern "C" {

const char *zxh_version(void) { return "zxh_b200 0.1.0 (sm_100a)"; }

int zxh_device_info(int device, char *name, size_t capacity, int *sms)
{
    if (device < 0) return ZXH_ERR_ARG;
    cudaDeviceProp prop;
    const cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return ZXH_ERR_CUDA;
    if (name && capacity) {
        std::strncpy(name, prop.name, capacity - 1);
        name[capacity - 1] = '\0';
    }
    if (sms) *sms = prop.multiProcessorCount;
    return ZXH_OK;
}

const char *zxh_last_error(const zxh_sim *sim)
{
    if (!sim) return g_create_error.c_str();
    return sim->err.c_str();
}

int zxh_create(zxh_sim **out, size_t n, int disable_x, int eager_expand_all, int dtype, int device)
{
    if (!out) return fail(nullptr, ZXH_ERR_ARG, "out is null");
    *out = nullptr;
    if (n < 1 || n > 63) return fail(nullptr, ZXH_ERR_LIMIT, "n must be in 1..63");
    if (dtype != ZXH_C64 && dtype != ZXH_C128) return fail(nullptr, ZXH_ERR_ARG, "dtype must be ZXH_C64 or ZXH_C128");
    zxh_sim *s = new (std::nothrow) zxh_sim();
    if (!s) return fail(nullptr, ZXH_ERR_OOM, "out of host memory");
    s->n = n;
    s->disable_x = disable_x != 0;
    s->eager = eager_expand_all != 0;
    s->dtype = dtype;
    s->elem_bytes = dtype == ZXH_C64 ? 8 : 16;
    s->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&s->d_status), sizeof(zxh::DevStatus));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&s->h_status), sizeof(zxh::DevStatus));
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
    if (e != cudaSuccess) {
        const std::string msg = std::string("CUDA init: ") + cudaGetErrorString(e);
        zxh_destroy(s);
        return fail(nullptr, ZXH_ERR_CUDA, msg);
    }
    s->ws.map.reset(int(n));
    *out = s;
    return ZXH_OK;
}

int zxh_destroy(zxh_sim *s)
{
    if (!s) return ZXH_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->d_state) cudaFree(s->d_state);
    if (s->d_blob) cudaFree(s->d_blob);
    if (s->h_stage) cudaFreeHost(s->h_stage);
    if (s->d_status) cudaFree(s->d_status);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->d_samp) cudaFree(s->d_samp);
    if (s->d_cnt) cudaFree(s->d_cnt);
    for (int j = 0; j < 2; j++) {
        if (s->h_async[j]) cudaFreeHost(s->h_async[j]);
        if (s->async_ev[j]) cudaEventDestroy(s->async_ev[j]);
    }
    if (s->d_out) cudaFree(s->d_out);
    if (s->d_psi) cudaFree(s->d_psi);
    if (s->d_lam) cudaFree(s->d_lam);
    if (s->d_ckpt) cudaFree(s->d_ckpt);
    if (s->d_adj) cudaFree(s->d_adj);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->evf0) cudaEventDestroy(s->evf0);
    if (s->evf1) cudaEventDestroy(s->evf1);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return ZXH_OK;
}

int zxh_set_seed(zxh_sim *s, uint64_t seed)
{
    if (!s) return ZXH_ERR_ARG;
    s->use_seed = true;
    s->seed = seed;
    return ZXH_OK;
}

int zxh_clear_seed(zxh_sim *s)
{
    if (!s) return ZXH_ERR_ARG;
    s->use_seed = false;
    s->seed = 0;
    return ZXH_OK;
}

int zxh_clear_gates(zxh_sim *s)
{
    if (!s) return ZXH_ERR_ARG;
    s->gates.clear();
    s->ws.gphase = zxh::cd(1.0, 0.0);  // zxh.cpp:228-232
    return ZXH_OK;
}

int zxh_barrier(zxh_sim *s) { return s ? push(s, zxh::G_BARRIER, 0, 0, 0, 0, 0) : ZXH_ERR_ARG; }

int zxh_rz(zxh_sim *s, size_t q, double theta)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "Rz")) return rc;
    return push(s, zxh::G_RZ, 0, q, theta, 0, 0);
}

int zxh_crz(zxh_sim *s, size_t cq, size_t q, double theta)
{
    if (!s) return ZXH_ERR_ARG;
    if (cq >= s->n || q >= s->n) return fail(s, ZXH_ERR_ARG, "CRz qubit out of range");
    push(s, zxh::G_P, 0, cq, -0.5 * theta, 0, 0);  // zxh.cpp:246-252
    return push(s, zxh::G_CP, cq, q, theta, 0, 0);
}

int zxh_cp(zxh_sim *s, size_t cq, size_t q, double theta)
{
    if (!s) return ZXH_ERR_ARG;
    if (cq >= s->n || q >= s->n) return fail(s, ZXH_ERR_ARG, "CP qubit out of range");
    return push(s, zxh::G_CP, cq, q, theta, 0, 0);
}

int zxh_p(zxh_sim *s, size_t q, double theta)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "P")) return rc;
    return push(s, zxh::G_P, 0, q, theta, 0, 0);
}

int zxh_z(zxh_sim *s, size_t q)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "Z")) return rc;
    return push(s, zxh::G_Z, 0, q, 0, 0, 0);
}

int zxh_x(zxh_sim *s, size_t q)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "X")) return rc;
    return push(s, zxh::G_X, 0, q, 0, 0, 0);
}

int zxh_cx(zxh_sim *s, size_t cq, size_t q)
{
    if (!s) return ZXH_ERR_ARG;
    if (cq >= s->n || q >= s->n) return fail(s, ZXH_ERR_ARG, "CX qubit out of range");
    return push(s, zxh::G_CX, cq, q, 0, 0, 0);
}

int zxh_h(zxh_sim *s, size_t q)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "H")) return rc;
    return push(s, zxh::G_H, 0, q, 0, 0, 0);
}

int zxh_u3(zxh_sim *s, size_t q, double theta, double lambda, double phi)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "U3")) return rc;
    return push(s, zxh::G_U3, 0, q, theta, lambda, phi);
}

int zxh_rx(zxh_sim *s, size_t q, double theta)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = check_q(s, q, "Rx")) return rc;
    return push(s, zxh::G_U3, 0, q, theta, kPi / 2.0, -kPi / 2.0);  // zxh.cpp:303-310
}

int zxh_push_gates(zxh_sim *s, const zxh_gate *gates, size_t count)
{
    if (!s) return ZXH_ERR_ARG;
    if (count && !gates) return fail(s, ZXH_ERR_ARG, "gates is null");
    std::vector<Gate> tmp;
    tmp.reserve(count + count / 8);
    for (size_t i = 0; i < count; i++)
        if (int rc = lower(s, gates[i], tmp)) return rc;
    s->gates.insert(s->gates.end(), tmp.begin(), tmp.end());
    return ZXH_OK;
}

int zxh_execute(zxh_sim *s)
{
    if (!s) return ZXH_ERR_ARG;
    if (int rc = use_device(s)) return rc;
    const int M = s->eager ? int(s->n) : zxh::calc_mem(s->gates.data(), s->gates.size(), int(s->n), s->disable_x);
    const size_t need = size_t(s->elem_bytes) << M;
    if (int rc = ensure_dev(s, &s->d_state, s->state_cap_bytes, std::max<size_t>(need, 256), "cudaMalloc(state)"))
        return rc;
    s->M = M;
    s->executed = false;
    s->measured = 0;
    s->pending.clear();  // the state restarts from |0...0>
    zxh::WalkState &ws = s->ws;
    ws.map.reset(int(s->n));
    ws.m = 0;
    ws.gphase = zxh::cd(1.0, 0.0);
    ws.fresh = true;
    ws.init_bits = 0;
    if (s->eager) {  // expand_all, zxh.cpp:721-729
        for (size_t q = 0; q < s->n; q++) ws.map.append_col(int(q));
        ws.m = int(s->n);
        ws.init_bits = int(s->n);
    }
    zxh::WalkState start = ws;
    std::vector<zxh::Op> ops;
    std::string err;
    if (int rc = zxh::walk(s->gates.data(), s->gates.size(), s->disable_x, M, ws, ops, err)) return fail(s, rc, err);
    zxh::Plan pl;
    if (int rc = zxh::plan(ops, s->elem_bytes, s->pp, start, pl, err)) return fail(s, rc, err);
    if (int rc = run_plan(s, pl)) return rc;
    ws.fresh = false;
    s->executed = true;
    return ZXH_OK;
}

// Host planning of one batch (zxh_apply and zxh_apply_async): the plan, the walk
// state after it and the phases it leaves over. The phases the previous batch left
// over ride in this batch's first window (or run first, on their own).
static int plan_batch(zxh_sim *s, const zxh_gate *gates, size_t count, zxh::Plan &pl, zxh::WalkState &ws,
                      std::vector<zxh::DiagTerm> &left)
{
    std::vector<Gate> tmp;
    for (size_t i = 0; i < count; i++)
        if (int rc = lower(s, gates[i], tmp)) return rc;
    zxh::WalkState start = s->ws;
    ws = s->ws;
    std::vector<zxh::Op> ops;
    std::string err;
    if (int rc = zxh::walk(tmp.data(), tmp.size(), s->disable_x, s->M, ws, ops, err)) return fail(s, rc, err);
    if (int rc = zxh::plan(ops, s->elem_bytes, s->pp, start, pl, err, &s->pending, &left)) return fail(s, rc, err);
    return ZXH_OK;
}

int zxh_apply(zxh_sim *s, const zxh_gate *gates, size_t count)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "zxh_apply requires zxh_execute first");
    if (count && !gates) return fail(s, ZXH_ERR_ARG, "gates is null");
    if (int rc = use_device(s)) return rc;
    zxh::Plan pl;
    zxh::WalkState ws;
    std::vector<zxh::DiagTerm> left;
    if (int rc = plan_batch(s, gates, count, pl, ws, left)) return rc;
    if (int rc = run_plan(s, pl)) return rc;
    s->ws = ws;
    s->pending = std::move(left);
    s->measured = 0;
    return ZXH_OK;
}

int zxh_apply_async(zxh_sim *s, const zxh_gate *gates, size_t count)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "zxh_apply_async requires zxh_execute first");
    if (count && !gates) return fail(s, ZXH_ERR_ARG, "gates is null");
    CK(s, cudaSetDevice(s->device), "cudaSetDevice");
    zxh::Plan pl;
    zxh::WalkState ws;
    std::vector<zxh::DiagTerm> left;
    if (int rc = plan_batch(s, gates, count, pl, ws, left)) return rc;  // overlaps the steps in flight
    const size_t bytes = std::max<size_t>(pl.blob.size(), 16);
    if (bytes > s->async_cap || bytes > s->blob_cap) {
        // growing a buffer that queued work may still read: settle first
        if (int rc = zxh_sync(s)) return rc;
        if (bytes > s->async_cap) {
            for (int j = 0; j < 2; j++) {
                if (s->h_async[j]) cudaFreeHost(s->h_async[j]);
                s->h_async[j] = nullptr;
            }
            s->async_cap = 0;
            for (int j = 0; j < 2; j++)
                CK(s, cudaMallocHost(reinterpret_cast<void **>(&s->h_async[j]), bytes * 2), "cudaMallocHost(program)");
            s->async_cap = bytes * 2;
        }
        if (int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_blob), s->blob_cap, bytes * 2,
                                "cudaMalloc(program)"))
            return rc;
    }
    const int j = s->async_slot;
    if (!s->async_ev[j]) CK(s, cudaEventCreateWithFlags(&s->async_ev[j], cudaEventDisableTiming), "event");
    CK(s, cudaEventSynchronize(s->async_ev[j]), "program slot");  // the upload that last read slot j has run
    std::memcpy(s->h_async[j], pl.blob.data(), pl.blob.size());
    if (!s->async_pending)  // a step's failure stays recorded until zxh_sync reads it
        CK(s, cudaMemsetAsync(s->d_status, 0, sizeof(zxh::DevStatus), s->stream), "reset status");
    CK(s, cudaMemcpyAsync(s->d_blob, s->h_async[j], pl.blob.size(), cudaMemcpyHostToDevice, s->stream),
       "upload program");
    CK(s, cudaEventRecord(s->async_ev[j], s->stream), "event");
    uint64_t kernels = 0;
    CK(s, zxh::run_passes(pl.passes, s->d_blob, s->d_state, s->elem_bytes, s->d_status, s->sms, s->stream, kernels),
       "launch");
    CK(s, cudaMemcpyAsync(s->h_status, s->d_status, sizeof(zxh::DevStatus), cudaMemcpyDeviceToHost, s->stream),
       "read status");
    s->async_slot ^= 1;
    s->async_pending = true;
    s->stat_kernels = kernels;
    s->stat_passes = 0;
    for (const zxh::Pass &p : pl.passes)
        if (p.kind != zxh::Pass::PRODUCT) s->stat_passes++;
    s->last_ms = 0.0f;
    s->ws = ws;
    s->pending = std::move(left);
    s->measured = 0;
    return ZXH_OK;
}

int zxh_flush(zxh_sim *s)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "zxh_flush requires zxh_execute first");
    if (int rc = use_device(s)) return rc;
    s->stat_kernels = 0;
    s->stat_passes = 0;
    s->last_ms = 0.0f;
    return flush_pending(s);
}

int zxh_sync(zxh_sim *s)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->async_pending) return ZXH_OK;
    s->async_pending = false;
    CK(s, cudaStreamSynchronize(s->stream), "apply_async");
    if (s->h_status->code != 0)
        return fail(s, int(s->h_status->code),
                    "device wait gave up (site " + std::to_string(s->h_status->where) + ")");
    return ZXH_OK;
}

int zxh_measure(zxh_sim *s, size_t shots)
{
    if (!s) return ZXH_ERR_ARG;
    if (shots == 0) {
        s->measured = 0;
        return ZXH_OK;
    }
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "measure requires execute() to be called first");
    if (shots > (size_t(1) << 40)) return fail(s, ZXH_ERR_LIMIT, "too many shots");
    if (int rc = use_device(s)) return rc;
    if (int rc = flush_pending(s)) return rc;
    const uint64_t base = s->use_seed ? s->seed : uint64_t(std::random_device{}());  // measure_cuda.cu:111-116
    const uint64_t stream_seed = zxh::mix_seed_host(base, 0);                        // measure_cuda.cu:1033
    const int m = s->ws.m;
    const uint64_t local = 1ULL << m;
    const uint64_t seglen = std::min<uint64_t>(4096, local);
    const uint64_t nseg = local / seglen;
    const size_t need = zxh::SamplerScratch::need_bytes(nseg, shots, true);
    if (int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_samp), s->samp_cap, need, "cudaMalloc(sampler)"))
        return rc;
    s->sc.carve(s->d_samp, nseg, shots, true);
    static thread_local uint64_t tab[8][256];
    column_tables(s->ws.map, tab);
    CK(s, cudaMemsetAsync(s->d_status, 0, sizeof(zxh::DevStatus), s->stream), "reset status");
    uint64_t kernels = 0;
    CK(s, cudaEventRecord(s->ev0, s->stream), "event");
    CK(s, zxh::run_sampler(s->d_state, s->elem_bytes, m, shots, stream_seed, &tab[0][0], s->ws.map.b(), s->sc,
                           s->d_status, s->sms, s->stream, kernels),
       "sampler launch");
    CK(s, cudaEventRecord(s->ev1, s->stream), "event");
    CK(s, cudaMemcpyAsync(s->h_status, s->d_status, sizeof(zxh::DevStatus), cudaMemcpyDeviceToHost, s->stream),
       "read status");
    CK(s, cudaStreamSynchronize(s->stream), "sampler");
    CK(s, cudaEventElapsedTime(&s->last_ms, s->ev0, s->ev1), "event time");
    s->stat_kernels = kernels;
    s->stat_passes = 2;
    if (s->h_status->code != 0) return fail(s, int(s->h_status->code), "sampler device wait gave up");
    s->measured = shots;
    s->measured_m = m;
    s->cnt_ready = false;
    return ZXH_OK;
}

int zxh_get_results(zxh_sim *s, uint64_t *words, size_t shots)
{
    if (!s) return ZXH_ERR_ARG;
    if (shots == 0) return ZXH_OK;
    if (!words) return fail(s, ZXH_ERR_ARG, "get_results results is null");
    if (shots > s->measured) return fail(s, ZXH_ERR_ARG, "get_results count exceeds cached result count");
    if (int rc = use_device(s)) return rc;
    CK(s, cudaMemcpyAsync(words, s->sc.words, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream),
       "copy results");
    CK(s, cudaStreamSynchronize(s->stream), "copy results");
    return ZXH_OK;
}

int zxh_counts(zxh_sim *s, uint64_t *words, uint64_t *counts, size_t capacity, size_t *n_unique)
{
    if (!s || !n_unique) return ZXH_ERR_ARG;
    *n_unique = 0;
    if (s->measured == 0) return ZXH_OK;
    if (words && !counts) return fail(s, ZXH_ERR_ARG, "counts: counts is null");
    if (int rc = use_device(s)) return rc;
    const int m = s->measured_m;
    const uint64_t nseg = (1ULL << m) / std::min<uint64_t>(4096, 1ULL << m);
    const size_t seg_bytes = (nseg * 8 + 255) & ~size_t(255);
    const size_t shot_bytes = (s->measured * 8 + 255) & ~size_t(255);
    const size_t need = 2 * seg_bytes + 256 + 2 * shot_bytes;
    uint64_t kernels = 0;
    if (!s->cnt_ready) {
        if (int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_cnt), s->cnt_cap, need, "cudaMalloc(counts)"))
            return rc;
    }
    auto *nuniq = reinterpret_cast<unsigned long long *>(s->d_cnt);
    auto *uoff = reinterpret_cast<unsigned long long *>(s->d_cnt + seg_bytes);
    auto *total = reinterpret_cast<unsigned long long *>(s->d_cnt + 2 * seg_bytes);
    auto *dwords = reinterpret_cast<uint64_t *>(s->d_cnt + 2 * seg_bytes + 256);
    auto *dhits = reinterpret_cast<uint64_t *>(s->d_cnt + 2 * seg_bytes + 256 + shot_bytes);
    CK(s, cudaEventRecord(s->ev0, s->stream), "event");
    if (!s->cnt_ready) {
        CK(s, zxh::run_counts(s->sc, m, s->ws.map.b(), nuniq, uoff, total, dwords, dhits, 1, s->sms, s->stream,
                              kernels),
           "counts launch");
        CK(s, cudaMemcpyAsync(&s->cnt_total, total, sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream),
           "read count total");
        CK(s, cudaStreamSynchronize(s->stream), "counts");
        s->cnt_ready = true;
    }
    *n_unique = size_t(s->cnt_total);
    if (!words) {
        CK(s, cudaEventRecord(s->ev1, s->stream), "event");
        CK(s, cudaStreamSynchronize(s->stream), "counts");
        CK(s, cudaEventElapsedTime(&s->last_ms, s->ev0, s->ev1), "event time");
        s->stat_kernels = kernels;
        s->stat_passes = 0;
        return ZXH_OK;
    }
    if (capacity < s->cnt_total) return fail(s, ZXH_ERR_LIMIT, "counts: capacity below the number of distinct outcomes");
    CK(s, zxh::run_counts(s->sc, m, s->ws.map.b(), nuniq, uoff, total, dwords, dhits, 2, s->sms, s->stream, kernels),
       "counts launch");
    CK(s, cudaEventRecord(s->ev1, s->stream), "event");
    CK(s, cudaMemcpyAsync(words, dwords, s->cnt_total * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream),
       "copy count words");
    CK(s, cudaMemcpyAsync(counts, dhits, s->cnt_total * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream),
       "copy counts");
    CK(s, cudaStreamSynchronize(s->stream), "counts");
    CK(s, cudaEventElapsedTime(&s->last_ms, s->ev0, s->ev1), "event time");
    s->stat_kernels = kernels;
    s->stat_passes = 0;
    return ZXH_OK;
}

int zxh_measured_count(const zxh_sim *s, size_t *out)
{
    if (!s || !out) return ZXH_ERR_ARG;
    *out = s->measured;
    return ZXH_OK;
}

static int state_to_device(zxh_sim *s, void *dst, int order)
{
    const int N = int(s->n);
    const uint64_t nv = 1ULL << N;
    if (s->ws.m < N) CK(s, cudaMemsetAsync(dst, 0, size_t(nv) * size_t(s->elem_bytes), s->stream), "zero state");
    static thread_local uint64_t tab[8][256];
    column_tables(s->ws.map, tab);
    void *dtab = nullptr;
    CK(s, cudaMallocAsync(&dtab, sizeof(tab), s->stream), "cudaMallocAsync(table)");
    CK(s, cudaMemcpyAsync(dtab, tab, sizeof(tab), cudaMemcpyHostToDevice, s->stream), "upload table");
    CK(s, zxh::run_scatter(s->d_state, 1ULL << s->ws.m, static_cast<uint64_t *>(dtab), s->ws.map.b(), N, order,
                           s->ws.gphase.real(), s->ws.gphase.imag(), dst, s->elem_bytes, s->sms, s->stream),
       "scatter");
    CK(s, cudaFreeAsync(dtab, s->stream), "cudaFreeAsync(table)");
    return ZXH_OK;
}

int zxh_get_state(zxh_sim *s, void *out, size_t out_elems, int order)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "get_state requires execute() to be called first");
    if (!out) return fail(s, ZXH_ERR_ARG, "out is null");
    if (s->n > 40) return fail(s, ZXH_ERR_LIMIT, "get_state export needs fewer than 41 qubits");
    const uint64_t nv = 1ULL << s->n;
    if (out_elems < nv) return fail(s, ZXH_ERR_ARG, "output buffer holds fewer than 2^n amplitudes");
    if (int rc = use_device(s)) return rc;
    if (int rc = flush_pending(s)) return rc;
    const size_t bytes = size_t(nv) * size_t(s->elem_bytes);
    if (int rc = ensure_dev(s, &s->d_out, s->out_cap, bytes, "cudaMalloc(get_state)")) return rc;
    if (int rc = state_to_device(s, s->d_out, order)) return rc;
    CK(s, cudaMemcpyAsync(out, s->d_out, bytes, cudaMemcpyDeviceToHost, s->stream), "copy state");
    CK(s, cudaStreamSynchronize(s->stream), "get_state");
    return ZXH_OK;
}

int zxh_get_state_device(zxh_sim *s, void *out_device, size_t out_elems, int order)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "get_state requires execute() to be called first");
    if (!out_device) return fail(s, ZXH_ERR_ARG, "out is null");
    if (s->n > 40) return fail(s, ZXH_ERR_LIMIT, "get_state export needs fewer than 41 qubits");
    if (out_elems < (1ULL << s->n)) return fail(s, ZXH_ERR_ARG, "output buffer holds fewer than 2^n amplitudes");
    if (int rc = use_device(s)) return rc;
    if (int rc = flush_pending(s)) return rc;
    if (int rc = state_to_device(s, out_device, order)) return rc;
    CK(s, cudaStreamSynchronize(s->stream), "get_state");
    return ZXH_OK;
}

int zxh_required_M(const zxh_sim *s, size_t *out)
{
    if (!s || !out) return ZXH_ERR_ARG;
    *out = size_t(zxh::calc_mem(s->gates.data(), s->gates.size(), int(s->n), s->disable_x));
    return ZXH_OK;
}

int zxh_num_qubits(const zxh_sim *s, size_t *out)
{
    if (!s || !out) return ZXH_ERR_ARG;
    *out = s->n;
    return ZXH_OK;
}

int zxh_state_view(zxh_sim *s, void **data, size_t *m_bits, size_t *elem_bytes, double *gre, double *gim)
{
    if (!s) return ZXH_ERR_ARG;
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "state_view requires execute() first");
    if (!s->pending.empty()) {  // the state as it stands, with the phases the last apply left over
        if (int rc = use_device(s)) return rc;
        if (int rc = flush_pending(s)) return rc;
    }
    if (data) *data = s->d_state;
    if (m_bits) *m_bits = size_t(s->ws.m);
    if (elem_bytes) *elem_bytes = size_t(s->elem_bytes);
    if (gre) *gre = s->ws.gphase.real();
    if (gim) *gim = s->ws.gphase.imag();
    return ZXH_OK;
}

int zxh_stream(zxh_sim *s, void **stream)
{
    if (!s || !stream) return ZXH_ERR_ARG;
    *stream = s->stream;
    return ZXH_OK;
}

int zxh_plan_stats(size_t n, int disable_x, int eager_expand_all, int dtype, const zxh_gate *gates, size_t count,
                   uint64_t *out)
{
    if (!out || (count && !gates)) return fail(nullptr, ZXH_ERR_ARG, "null argument");
    if (n < 1 || n > 63) return fail(nullptr, ZXH_ERR_LIMIT, "n must be in 1..63");
    if (dtype != ZXH_C64 && dtype != ZXH_C128) return fail(nullptr, ZXH_ERR_ARG, "dtype must be ZXH_C64 or ZXH_C128");
    zxh_sim tmp;  // host fields only; no CUDA call is made
    tmp.n = n;
    std::vector<Gate> gl;
    for (size_t i = 0; i < count; i++)
        if (int rc = lower(&tmp, gates[i], gl)) return fail(nullptr, rc, tmp.err);
    const int eb = dtype == ZXH_C64 ? 8 : 16;
    const int M = eager_expand_all ? int(n) : zxh::calc_mem(gl.data(), gl.size(), int(n), disable_x != 0);
    zxh::WalkState ws;
    ws.map.reset(int(n));
    if (eager_expand_all) {
        for (size_t q = 0; q < n; q++) ws.map.append_col(int(q));
        ws.m = int(n);
        ws.init_bits = int(n);
    }
    const zxh::WalkState start = ws;
    std::vector<zxh::Op> ops;
    std::string err;
    if (int rc = zxh::walk(gl.data(), gl.size(), disable_x != 0, M, ws, ops, err)) return fail(nullptr, rc, err);
    zxh::Plan pl;
    if (int rc = zxh::plan(ops, eb, tmp.pp, start, pl, err)) return fail(nullptr, rc, err);
    for (int k = 0; k < 13; k++) out[k] = 0;
    out[0] = uint64_t(M);
    out[1] = uint64_t(ws.m);
    for (const zxh::Pass &p : pl.passes) {
        if (p.kind == zxh::Pass::WALSH || p.kind == zxh::Pass::SPAN) {
            out[p.kind == zxh::Pass::WALSH ? 11 : 12]++;
            out[10]++;
            continue;
        }
        if (p.kind > zxh::Pass::GROW) continue;
        out[2 + int(p.kind)]++;
        if (p.kind != zxh::Pass::PRODUCT) out[10]++;
    }
    return ZXH_OK;
}

int zxh_set_param(zxh_sim *s, const char *name, int value)
{
    if (!s || !name) return ZXH_ERR_ARG;
    struct Entry { const char *key; int *field; int lo, hi; };
    const Entry table[] = {
        {"tile_bits_c64", &s->pp.tile_bits_c64, 1, 13},
        {"tile_bits_c128", &s->pp.tile_bits_c128, 1, 12},
        {"contig_bits", &s->pp.contig_bits, 1, 12},
        {"max_gates", &s->pp.max_gates, 1, 16},
        {"fast_gates", &s->pp.fast_gates, 1, 16},
        {"fast_fuse_quad", &s->pp.fast_fuse_quad, 0, 64},
        {"fast_contig_c64", &s->pp.fast_contig_c64, 1, 11},
        {"fast_contig_c128", &s->pp.fast_contig_c128, 0, 10},
        {"row_wide_c64", &s->pp.row_wide_c64, 0, 1},
        {"row_wide_c128", &s->pp.row_wide_c128, 0, 1},
        {"low_pass", &s->pp.low_pass, 0, 1},
        {"low_regs_c64", &s->pp.low_regs_c64, 0, 5},
        {"low_regs_c128", &s->pp.low_regs_c128, 0, 4},
        {"real_split", &s->pp.real_split, 0, 1},
        {"diag_prefetch_c64", &s->pp.diag_prefetch_c64, 0, 1},
        {"adj_regs", &s->pp.adj_regs, 1, 4},
        {"grow_staged", &s->pp.grow_staged, 0, 7},
        {"diag_prefetch_c128", &s->pp.diag_prefetch_c128, 0, 1},
        {"walsh", &s->pp.walsh, 0, 1},
        {"walsh_min_general", &s->pp.walsh_min_general, 0, 1 << 20},
        {"span", &s->pp.span, 0, 1},
        {"span_min_run", &s->pp.span_min_run, 3, 8},
        {"span_land", &s->pp.span_land, 0, 1},
        {"span_split", &s->pp.span_split, 0, 2},
        {"span_order", &s->pp.span_order, 0, 2},
        {"span_mixed", &s->pp.span_mixed, 0, 1},
        {"diag_chunk_bits", &s->pp.diag_chunk_bits, -1, 8},
        {"grow", &s->pp.grow, 0, 1},
        {"grow_regs", &s->pp.grow_regs, 1, 4},
        {"grow_only", &s->pp.grow_only, 0, 1},
        {"adj_windows", &s->pp.adj_windows, 0, 1},
        {"diag_row_bits_c64", &s->pp.diag_row_bits_c64, 2, 4},
        {"diag_row_bits_c128", &s->pp.diag_row_bits_c128, 2, 4},
    };
    for (const Entry &e : table)
        if (std::strcmp(e.key, name) == 0) {
            if (value < e.lo || value > e.hi)
                return fail(s, ZXH_ERR_ARG, std::string(name) + " must be in [" + std::to_string(e.lo) + ", " +
                                                std::to_string(e.hi) + "]");
            *e.field = value;
            return ZXH_OK;
        }
    return fail(s, ZXH_ERR_ARG, std::string("unknown parameter ") + name);
}

int zxh_last_stats(const zxh_sim *s, uint64_t *kernels, uint64_t *passes, double *device_ms)
{
    if (!s) return ZXH_ERR_ARG;
    if (kernels) *kernels = s->stat_kernels;
    if (passes) *passes = s->stat_passes;
    if (device_ms) *device_ms = double(s->last_ms);
    return ZXH_OK;
}

}  // extern "C"
