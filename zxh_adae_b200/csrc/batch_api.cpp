// batch_api.cpp -- zxh_batch_*: energies and adjoint gradients of many independent
// circuits (uneven qubit counts, one observable each) in one persistent launch,
// optionally replayed from a captured CUDA graph, with an autotuner over the
// pass shape and the task size.
//
// No counterpart in the reference (one circuit per ZXH object; its diagonal
// buckets and U3 descriptors are process-global, kernel_cuda.cu:91-142).
//
// Each circuit is compiled on the host with the same walk, planner and reverse
// program as zxh_adjoint_gradient, restricted to the pass set of the batch
// kernel: |0...0> init, general strided passes (windows fused, or alone as a
// pass without gates), lambda = H psi with the energy, general strided adjoint
// passes and adjoint diagonal groups. Every circuit's state and lambda live in
// one arena. The task queue lists the ops level by level (op k of every circuit,
// then op k + 1 ...), so an op's tasks always follow those of the op it waits for.
#include "adjoint_host.h"
#include "batch.h"
#include "sim.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace zxh::api;
using zxh::BatchOp;
using zxh::BatchTask;

struct zxh_batch {
    int device = 0, dtype = ZXH_C64, eb = 8, sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;

    std::vector<uint32_t> n;
    std::vector<std::vector<Gate>> gates;  // lowered records
    std::vector<std::vector<zxh_term>> terms;
    std::vector<size_t> grad_off;          // count + 1

    std::vector<BatchOp> ops;
    std::vector<BatchTask> tasks;
    std::vector<uint32_t> rem_init;
    std::vector<uint8_t> blob;
    std::vector<std::vector<uint32_t>> chain;  // op indices per circuit, in order
    std::vector<std::vector<zxh::AdjDiagGate>> hgates;  // host copies for the per-op launches
    size_t arena_elems = 0;

    uint8_t *d_blob = nullptr;
    BatchOp *d_ops = nullptr;
    BatchTask *d_tasks = nullptr;
    uint32_t *d_rem = nullptr, *d_rem_init = nullptr, *d_next = nullptr;
    void *d_arena = nullptr;
    double *d_grads = nullptr, *d_energy = nullptr;
    zxh::DevStatus *d_status = nullptr, *h_status = nullptr;
    size_t cap_blob = 0, cap_ops = 0, cap_tasks = 0, cap_rem = 0, cap_arena = 0, cap_grads = 0;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;

    int grow_regs = 4, task_items = 128, task_elems = 1 << 17;
    int threads = 256;         // threads per CTA of the persistent kernel (the warps working on one task)
    int adj_regs = 3;          // register coordinates (gates with high deltas) per reverse pass
    int wait_limit_log2 = 31;  // a task's wait for its predecessor: 2^31 SM clocks (about a second)
    uint64_t bytes = 0;  // algorithmic state bytes of one run
    bool real = false;   // every strided op has real gates: the persistent kernel's real-gate form
    float last_ms = 0.0f;
};

namespace {

thread_local std::string g_batch_error;

int bfail(zxh_batch *b, int code, const std::string &msg)
{
    if (b) b->err = msg;
    else g_batch_error = msg;
    return code;
}

int bcuda(zxh_batch *b, cudaError_t e, const char *what)
{
    return bfail(b, e == cudaErrorMemoryAllocation ? ZXH_ERR_OOM : ZXH_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

#define BCK(b, call, what)                                   \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return bcuda(b, e_, what);    \
    } while (0)

int grow_dev(zxh_batch *b, void **p, size_t &cap, size_t need, const char *what)
{
    need = std::max<size_t>(need, 256);
    if (*p && need <= cap) return ZXH_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    BCK(b, cudaMalloc(p, need), what);
    cap = need;
    return ZXH_OK;
}

void drop_graph(zxh_batch *b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

uint64_t append(std::vector<uint8_t> &blob, const void *p, size_t n)
{
    const uint64_t off = (blob.size() + 255) & ~uint64_t(255);
    blob.resize(off + n + 16, 0);
    if (n) std::memcpy(blob.data() + off, p, n);
    return off;
}

// Host compile of every circuit into ops, tasks and one descriptor blob.
int compile(zxh_batch *b)
{
    b->ops.clear();
    b->rem_init.clear();
    b->blob.clear();
    b->chain.assign(b->n.size(), std::vector<uint32_t>());
    b->bytes = 0;
    b->hgates.clear();
    b->arena_elems = 0;
    zxh::PlanParams pp;
    pp.grow_only = 1;
    pp.grow_regs = b->grow_regs;
    pp.adj_regs = b->adj_regs;  // the persistent kernel runs reverse passes of at most 3 register coordinates
    std::vector<uint8_t> etab;
    zxh::exp_table(b->eb, etab);
    const uint64_t exp_off = append(b->blob, etab.data(), etab.size());

    for (size_t c = 0; c < b->n.size(); c++) {
        const int N = int(b->n[c]);
        zxh_sim tmp;  // host fields only: the walk, planner and reverse program read these
        tmp.n = size_t(N);
        tmp.elem_bytes = b->eb;
        tmp.dtype = b->dtype;
        tmp.gates = b->gates[c];
        tmp.pp = pp;
        zxh::WalkState ws;
        ws.map.reset(N);
        for (int q = 0; q < N; q++) ws.map.append_col(q);
        ws.m = N;
        ws.init_bits = N;
        const zxh::WalkState start = ws;
        std::vector<zxh::Op> wops;
        std::string err;
        if (int rc = zxh::walk(tmp.gates.data(), tmp.gates.size(), false, N, ws, wops, err))
            return bfail(b, rc, "circuit " + std::to_string(c) + ": " + err);
        zxh::Plan pl;
        if (int rc = zxh::plan(wops, b->eb, pp, start, pl, err))
            return bfail(b, rc, "circuit " + std::to_string(c) + ": " + err);
        const uint64_t base = append(b->blob, pl.blob.data(), pl.blob.size());
        const uint64_t psi = b->arena_elems, lam = psi + (uint64_t(1) << N);
        b->arena_elems = lam + (uint64_t(1) << N);
        auto push = [&](BatchOp op) {
            op.circuit = uint32_t(c);
            op.m = uint32_t(N);
            op.psi = psi;
            op.lam = lam;
            op.grad_base = uint32_t(b->grad_off[c]);
            op.energy = uint32_t(c);
            op.dep = b->chain[c].empty() ? zxh::kNoDep : b->chain[c].back();
            const uint64_t sb = uint64_t(b->eb) << N;  // one state
            b->bytes += op.kind == zxh::BOP_INIT ? sb : (op.kind == zxh::BOP_GROW || op.kind == zxh::BOP_LAMBDA) ? 2 * sb : 4 * sb;
            b->chain[c].push_back(uint32_t(b->ops.size()));
            b->ops.push_back(op);
        };
        for (const zxh::Pass &ps : pl.passes) {
            BatchOp op;
            std::memset(&op, 0, sizeof(op));
            if (ps.kind == zxh::Pass::INIT) {
                op.kind = zxh::BOP_INIT;
                op.units = uint64_t(1) << N;
            } else if (ps.kind == zxh::Pass::GROW) {
                op.kind = zxh::BOP_GROW;
                op.R = uint32_t(ps.gb.regs.size());
                op.units = ps.gb.dev.nitems;
                op.base = base;
                op.off0 = ps.off;
                op.off1 = ps.off2;
                op.aux = ps.gb.all_real() ? 1u : 0u;
            } else {
                return bfail(b, ZXH_ERR_ARG, "circuit " + std::to_string(c) +
                                                 " needs a pass the batched launch does not run (n >= 6 required)");
            }
            push(op);
        }
        // lambda and energy
        std::vector<zxh::TermDev> dt;
        if (int rc = zxh::adj::compile_terms(&tmp, b->terms[c].data(), b->terms[c].size(), ws.map, N, false, dt))
            return bfail(b, rc, "circuit " + std::to_string(c) + ": " + tmp.err);
        {
            BatchOp op;
            std::memset(&op, 0, sizeof(op));
            op.kind = zxh::BOP_LAMBDA;
            op.units = uint64_t(1) << N;
            op.off0 = append(b->blob, dt.data(), dt.size() * sizeof(zxh::TermDev));
            op.aux = uint32_t(dt.size());
            push(op);
        }
        // reverse sweep
        std::vector<zxh::adj::RevStep> steps;
        std::vector<zxh::AdjDiagGate> dg;
        std::vector<uint32_t> ds;
        const std::vector<size_t> ends = {tmp.gates.size()};
        if (int rc = zxh::adj::reverse_program(&tmp, ends, ws.map, steps, dg, ds, zxh::kBatchDiagMax))
            return bfail(b, rc, "circuit " + std::to_string(c) + ": " + tmp.err);
        const std::vector<uint8_t> gblob = zxh::adj::pack_grow(steps);
        const uint64_t gbase = append(b->blob, gblob.data(), gblob.size());
        for (const zxh::adj::RevStep &r : steps) {
            BatchOp op;
            std::memset(&op, 0, sizeof(op));
            if (r.kind == zxh::adj::RevStep::GROW) {
                op.kind = zxh::BOP_GROW_ADJ;
                op.R = uint32_t(r.gb.regs.size());
                op.units = r.gb.dev.nitems;
                op.base = gbase;
                op.off0 = r.off;
                op.off1 = r.toff;
                op.aux = r.gb.all_real() ? 1u : 0u;
            } else if (r.kind == zxh::adj::RevStep::DIAG) {
                op.kind = zxh::BOP_DIAG_ADJ;
                op.units = uint64_t(1) << N;
                op.off0 = append(b->blob, dg.data() + r.first, r.ng * sizeof(zxh::AdjDiagGate));
                op.off1 = append(b->blob, ds.data() + r.first, r.ng * sizeof(uint32_t));
                op.off2 = exp_off;
                op.aux = r.ng;
            } else {
                return bfail(b, ZXH_ERR_ARG, "circuit " + std::to_string(c) + ": state too small for the batched launch");
            }
            push(op);
        }
    }
    return ZXH_OK;
}

// The task queue, level by level: op k of every circuit, then op k + 1 ...
void make_tasks(zxh_batch *b)
{
    b->tasks.clear();
    size_t levels = 0;
    for (const auto &ch : b->chain) levels = std::max(levels, ch.size());
    b->rem_init.assign(b->ops.size(), 0);
    for (size_t L = 0; L < levels; L++)
        for (size_t c = 0; c < b->chain.size(); c++) {
            if (L >= b->chain[c].size()) continue;
            const uint32_t oi = b->chain[c][L];
            const BatchOp &op = b->ops[oi];
            const bool grow = op.kind == zxh::BOP_GROW || op.kind == zxh::BOP_GROW_ADJ;
            const uint64_t per = grow ? uint64_t(b->task_items) : uint64_t(b->task_elems);
            for (uint64_t s = 0; s < op.units; s += per) {
                BatchTask t;
                t.op = oi;
                t.pad = 0;
                t.begin = s;
                t.end = std::min(op.units, s + per);
                b->tasks.push_back(t);
                b->rem_init[oi]++;
            }
        }
}

int upload(zxh_batch *b)
{
    drop_graph(b);
    const size_t ngr = b->grad_off.back();
    if (int rc = grow_dev(b, reinterpret_cast<void **>(&b->d_blob), b->cap_blob, b->blob.size(), "cudaMalloc(batch blob)"))
        return rc;
    if (int rc = grow_dev(b, reinterpret_cast<void **>(&b->d_ops), b->cap_ops, b->ops.size() * sizeof(BatchOp),
                          "cudaMalloc(batch ops)"))
        return rc;
    if (int rc = grow_dev(b, reinterpret_cast<void **>(&b->d_tasks), b->cap_tasks, b->tasks.size() * sizeof(BatchTask),
                          "cudaMalloc(batch tasks)"))
        return rc;
    if (int rc = grow_dev(b, reinterpret_cast<void **>(&b->d_rem), b->cap_rem,
                          (2 * b->ops.size() + 64) * sizeof(uint32_t), "cudaMalloc(batch counters)"))
        return rc;
    b->d_rem_init = b->d_rem + b->ops.size();
    b->d_next = b->d_rem + 2 * b->ops.size();
    if (int rc = grow_dev(b, &b->d_arena, b->cap_arena, b->arena_elems * size_t(b->eb), "cudaMalloc(batch states)"))
        return rc;
    if (int rc = grow_dev(b, reinterpret_cast<void **>(&b->d_grads), b->cap_grads,
                          (ngr + b->n.size() + 64) * sizeof(double), "cudaMalloc(batch gradients)"))
        return rc;
    b->d_energy = b->d_grads + ngr;
    BCK(b, cudaMemcpyAsync(b->d_blob, b->blob.data(), b->blob.size(), cudaMemcpyHostToDevice, b->stream), "upload blob");
    BCK(b, cudaMemcpyAsync(b->d_ops, b->ops.data(), b->ops.size() * sizeof(BatchOp), cudaMemcpyHostToDevice, b->stream),
        "upload ops");
    BCK(b, cudaMemcpyAsync(b->d_tasks, b->tasks.data(), b->tasks.size() * sizeof(BatchTask), cudaMemcpyHostToDevice,
                           b->stream),
        "upload tasks");
    BCK(b, cudaMemcpyAsync(b->d_rem_init, b->rem_init.data(), b->rem_init.size() * sizeof(uint32_t),
                           cudaMemcpyHostToDevice, b->stream),
        "upload counters");
    BCK(b, cudaStreamSynchronize(b->stream), "upload");
    return ZXH_OK;
}

// The device work of one persistent run (also what the graph captures).
int enqueue_persistent(zxh_batch *b)
{
    const size_t ngr = b->grad_off.back();
    BCK(b, cudaMemsetAsync(b->d_grads, 0, (ngr + b->n.size()) * sizeof(double), b->stream), "reset gradients");
    BCK(b, cudaMemsetAsync(b->d_next, 0, sizeof(uint32_t), b->stream), "reset queue");
    BCK(b, cudaMemsetAsync(b->d_status, 0, sizeof(zxh::DevStatus), b->stream), "reset status");
    BCK(b, cudaMemcpyAsync(b->d_rem, b->d_rem_init, b->ops.size() * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                           b->stream),
        "reset counters");
    BCK(b, zxh::run_batch_persistent(b->d_blob, b->d_ops, b->d_tasks, uint32_t(b->tasks.size()), b->d_next, b->d_rem,
                                     b->d_arena, b->d_grads, b->d_energy, b->d_status, b->eb, b->real,
                                     b->threads, b->wait_limit_log2, b->sms, b->stream),
        "batch launch");
    return ZXH_OK;
}

// One op as its own launch of the library's regular pass kernels (the
// sequential comparison: one launch at a time).
int launch_op(zxh_batch *b, const BatchOp &op)
{
    uint8_t *arena = static_cast<uint8_t *>(b->d_arena);
    void *psi = arena + op.psi * uint64_t(b->eb);
    void *lam = arena + op.lam * uint64_t(b->eb);
    double *gr = b->d_grads + op.grad_base;
    cudaError_t e = cudaSuccess;
    switch (op.kind) {
    case zxh::BOP_INIT:
        e = cudaMemsetAsync(psi, 0, size_t(b->eb) << op.m, b->stream);
        if (e == cudaSuccess) e = zxh::run_set_one(psi, b->eb, b->stream);
        break;
    case zxh::BOP_GROW:
        e = zxh::run_grow(b->d_blob + op.base, op.off0, op.off1, int(op.R), op.units, b->eb, psi, nullptr, nullptr,
                          op.aux != 0, (zxh::PlanParams().grow_staged & 2) != 0, b->d_status, b->sms, b->stream);
        break;
    case zxh::BOP_LAMBDA:
        e = zxh::run_lambda(psi, lam, int(op.m), b->eb, reinterpret_cast<const zxh::TermDev *>(b->d_blob + op.off0),
                            op.aux, b->d_energy + op.energy, b->sms, b->stream);
        break;
    case zxh::BOP_GROW_ADJ:
        e = zxh::run_grow(b->d_blob + op.base, op.off0, op.off1, int(op.R), op.units, b->eb, psi, lam, gr,
                          op.aux != 0, (zxh::PlanParams().grow_staged & (b->eb == 8 ? 1 : 4)) != 0, b->d_status,
                          b->sms, b->stream);
        break;
    case zxh::BOP_DIAG_ADJ:
        e = zxh::run_adj_diag(psi, lam, int(op.m), b->eb,
                              reinterpret_cast<const zxh::AdjDiagGate *>(b->blob.data() + op.off0), op.aux, gr,
                              reinterpret_cast<const uint32_t *>(b->blob.data() + op.off1), b->d_blob + op.off2,
                              b->sms, b->stream);
        break;
    default: return bfail(b, ZXH_ERR_ARG, "unknown batch op");
    }
    BCK(b, e, "batch pass launch");
    return ZXH_OK;
}

int build(zxh_batch *b)
{
    if (int rc = compile(b)) return rc;
    b->real = true;
    for (const BatchOp &op : b->ops)
        if ((op.kind == zxh::BOP_GROW || op.kind == zxh::BOP_GROW_ADJ) && !op.aux) b->real = false;
    make_tasks(b);
    return upload(b);
}

// New task sizes only: the compiled ops stay, the queue is rebuilt.
int retask(zxh_batch *b)
{
    make_tasks(b);
    return upload(b);
}

}  // namespace

extern "C" {

const char *zxh_batch_last_error(const zxh_batch *b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

int zxh_batch_create(zxh_batch **out, size_t count, const uint32_t *nqubits, const size_t *gate_offsets,
                     const zxh_gate *gates, const size_t *term_offsets, const zxh_term *terms, int dtype, int device)
{
    if (!out) return bfail(nullptr, ZXH_ERR_ARG, "out is null");
    *out = nullptr;
    if (!count || !nqubits || !gate_offsets || !term_offsets) return bfail(nullptr, ZXH_ERR_ARG, "null argument");
    if (dtype != ZXH_C64 && dtype != ZXH_C128) return bfail(nullptr, ZXH_ERR_ARG, "dtype must be ZXH_C64 or ZXH_C128");
    zxh_batch *b = new (std::nothrow) zxh_batch();
    if (!b) return bfail(nullptr, ZXH_ERR_OOM, "out of host memory");
    b->device = device;
    b->dtype = dtype;
    b->eb = dtype == ZXH_C64 ? 8 : 16;
    b->grad_off.assign(1, 0);
    for (size_t c = 0; c < count; c++) {
        const uint32_t nq = nqubits[c];
        if (nq < 6 || nq > 34) {
            zxh_batch_destroy(b);
            return bfail(nullptr, ZXH_ERR_LIMIT, "batched circuits need 6..34 qubits");
        }
        zxh_sim tmp;
        tmp.n = nq;
        std::vector<Gate> low;
        for (size_t i = gate_offsets[c]; i < gate_offsets[c + 1]; i++)
            if (int rc = lower(&tmp, gates[i], low)) {
                const std::string msg = "circuit " + std::to_string(c) + ": " + tmp.err;
                zxh_batch_destroy(b);
                return bfail(nullptr, rc, msg);
            }
        b->n.push_back(nq);
        b->gates.push_back(low);
        b->grad_off.push_back(b->grad_off.back() + low.size());
        b->terms.emplace_back(terms + term_offsets[c], terms + term_offsets[c + 1]);
    }
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&b->d_status), sizeof(zxh::DevStatus));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&b->h_status), sizeof(zxh::DevStatus));
    if (e != cudaSuccess) {
        const std::string msg = std::string("CUDA init: ") + cudaGetErrorString(e);
        zxh_batch_destroy(b);
        return bfail(nullptr, ZXH_ERR_CUDA, msg);
    }
    if (int rc = build(b)) {
        const std::string msg = b->err;
        zxh_batch_destroy(b);
        return bfail(nullptr, rc, msg);
    }
    *out = b;
    return ZXH_OK;
}

int zxh_batch_destroy(zxh_batch *b)
{
    if (!b) return ZXH_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    void *ptrs[] = {b->d_blob, b->d_ops, b->d_tasks, b->d_rem, b->d_arena, b->d_grads, b->d_status};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->h_status) cudaFreeHost(b->h_status);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return ZXH_OK;
}

int zxh_batch_gradient_offsets(const zxh_batch *b, size_t *offsets)
{
    if (!b || !offsets) return ZXH_ERR_ARG;
    for (size_t i = 0; i < b->grad_off.size(); i++) offsets[i] = b->grad_off[i];
    return ZXH_OK;
}

int zxh_batch_run(zxh_batch *b, int mode, double *energies, double *grads, size_t ngrads)
{
    if (!b) return ZXH_ERR_ARG;
    const size_t ngr = b->grad_off.back();
    if ((ngr && !grads) || !energies) return bfail(b, ZXH_ERR_ARG, "output is null");
    if (ngrads < ngr) return bfail(b, ZXH_ERR_ARG, "grads holds fewer entries than the batch's recorded gates");
    if (mode < ZXH_BATCH_SEQUENTIAL || mode > ZXH_BATCH_GRAPH) return bfail(b, ZXH_ERR_ARG, "unknown batch mode");
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    if (mode == ZXH_BATCH_GRAPH && !b->gexec) {
        BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        const int rc = enqueue_persistent(b);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        BCK(b, ce, "end capture");
        b->graph = g;
        BCK(b, cudaGraphInstantiate(&b->gexec, b->graph, 0), "instantiate graph");
    }
    BCK(b, cudaEventRecord(b->ev0, b->stream), "event");
    if (mode == ZXH_BATCH_GRAPH) {
        BCK(b, cudaGraphLaunch(b->gexec, b->stream), "graph launch");
    } else if (mode == ZXH_BATCH_PERSISTENT) {
        if (int rc = enqueue_persistent(b)) return rc;
    } else {
        BCK(b, cudaMemsetAsync(b->d_grads, 0, (ngr + b->n.size()) * sizeof(double), b->stream), "reset gradients");
        BCK(b, cudaMemsetAsync(b->d_status, 0, sizeof(zxh::DevStatus), b->stream), "reset status");
        for (const auto &ch : b->chain)
            for (uint32_t oi : ch)
                if (int rc = launch_op(b, b->ops[oi])) return rc;
    }
    BCK(b, cudaEventRecord(b->ev1, b->stream), "event");
    BCK(b, cudaMemcpyAsync(b->h_status, b->d_status, sizeof(zxh::DevStatus), cudaMemcpyDeviceToHost, b->stream),
        "read status");
    BCK(b, cudaMemcpyAsync(energies, b->d_energy, b->n.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream),
        "read energies");
    if (ngr)
        BCK(b, cudaMemcpyAsync(grads, b->d_grads, ngr * sizeof(double), cudaMemcpyDeviceToHost, b->stream),
            "read gradients");
    BCK(b, cudaStreamSynchronize(b->stream), "batch run");
    BCK(b, cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1), "event time");
    if (b->h_status->code != 0)
        return bfail(b, int(b->h_status->code), "batch task wait gave up (site " + std::to_string(b->h_status->where) +
                                                     ", task " + std::to_string(b->h_status->info) + ")");
    return ZXH_OK;
}

int zxh_batch_set(zxh_batch *b, const char *name, int value)
{
    if (!b || !name) return ZXH_ERR_ARG;
    int *field = nullptr;
    int lo = 0, hi = 0;
    if (!std::strcmp(name, "grow_regs")) field = &b->grow_regs, lo = 1, hi = 4;
    else if (!std::strcmp(name, "task_items")) field = &b->task_items, lo = 1, hi = 1 << 20;
    else if (!std::strcmp(name, "task_elems")) field = &b->task_elems, lo = 256, hi = 1 << 26;
    else if (!std::strcmp(name, "wait_limit_log2")) field = &b->wait_limit_log2, lo = 0, hi = 31;
    else if (!std::strcmp(name, "threads")) field = &b->threads, lo = 64, hi = 256;
    else if (!std::strcmp(name, "adj_regs")) field = &b->adj_regs, lo = 1, hi = 3;
    else return bfail(b, ZXH_ERR_ARG, std::string("unknown batch parameter ") + name);
    if (value < lo || value > hi || (field == &b->threads && value != 64 && value != 128 && value != 256))
        return bfail(b, ZXH_ERR_ARG, std::string(name) + " must be in [" + std::to_string(lo) + ", " +
                                         std::to_string(hi) + "]" +
                                         (field == &b->threads ? " and one of 64, 128, 256" : ""));
    *field = value;
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    if (field == &b->wait_limit_log2 || field == &b->threads) {
        // launch parameters: only the captured graph holds the old value
        BCK(b, cudaStreamSynchronize(b->stream), "sync");
        drop_graph(b);
        return ZXH_OK;
    }
    return (field == &b->grow_regs || field == &b->adj_regs) ? build(b) : retask(b);
}

int zxh_batch_get(const zxh_batch *b, const char *name, int *value)
{
    if (!b || !name || !value) return ZXH_ERR_ARG;
    if (!std::strcmp(name, "grow_regs")) *value = b->grow_regs;
    else if (!std::strcmp(name, "task_items")) *value = b->task_items;
    else if (!std::strcmp(name, "task_elems")) *value = b->task_elems;
    else if (!std::strcmp(name, "wait_limit_log2")) *value = b->wait_limit_log2;
    else if (!std::strcmp(name, "threads")) *value = b->threads;
    else if (!std::strcmp(name, "adj_regs")) *value = b->adj_regs;
    else return ZXH_ERR_ARG;
    return ZXH_OK;
}

int zxh_batch_stats(const zxh_batch *b, uint64_t *ops, uint64_t *tasks, double *device_ms, uint64_t *bytes)
{
    if (!b) return ZXH_ERR_ARG;
    if (bytes) *bytes = b->bytes;
    if (ops) *ops = b->ops.size();
    if (tasks) *tasks = b->tasks.size();
    if (device_ms) *device_ms = double(b->last_ms);
    return ZXH_OK;
}

int zxh_batch_tune(zxh_batch *b, int reps)
{
    if (!b) return ZXH_ERR_ARG;
    if (reps < 1) reps = 1;
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    const size_t ngr = b->grad_off.back();
    std::vector<double> e(b->n.size()), g(std::max<size_t>(ngr, 1));
    // best of reps timed persistent runs (the first run of a setting warms up)
    auto timed = [&](double &t) -> int {
        t = 1e300;
        for (int k = 0; k <= reps; k++) {
            if (int rc = zxh_batch_run(b, ZXH_BATCH_PERSISTENT, e.data(), g.data(), g.size())) return rc;
            if (k) t = std::min(t, double(b->last_ms));
        }
        return ZXH_OK;
    };
    // 1. gate-fusion depth x task size at the current threads and reverse depth
    const int regs_c[] = {2, 3, 4};
    const int items_c[] = {32, 128, 512, 2048};
    double best = 1e300;
    int best_r = b->grow_regs, best_i = b->task_items;
    for (int r : regs_c) {
        b->grow_regs = r;
        if (int rc = compile(b)) return rc;
        for (int it : items_c) {
            b->task_items = it;
            b->task_elems = it * 1024;
            if (int rc = retask(b)) return rc;
            double t;
            if (int rc = timed(t)) return rc;
            if (t < best) best = t, best_r = r, best_i = it;
        }
    }
    b->grow_regs = best_r;
    b->task_items = best_i;
    b->task_elems = best_i * 1024;
    if (int rc = build(b)) return rc;
    // 2. threads per CTA (the warps that share a task) at that setting
    const int threads_c[] = {64, 128, 256};
    int best_n = b->threads;
    for (int nt : threads_c) {
        if (nt == best_n) continue;
        const int keep = b->threads;
        b->threads = nt;
        double t;
        if (int rc = timed(t)) return rc;
        if (t < best) best = t, best_n = nt;
        b->threads = keep;
    }
    b->threads = best_n;
    // 3. register coordinates per reverse pass (fewer: more passes, less register pressure)
    int best_a = b->adj_regs;
    for (int a = 1; a <= 3; a++) {
        if (a == best_a) continue;
        const int keep = b->adj_regs;
        b->adj_regs = a;
        if (int rc = build(b)) return rc;
        double t;
        if (int rc = timed(t)) return rc;
        if (t < best) best = t, best_a = a;
        b->adj_regs = keep;
    }
    b->adj_regs = best_a;
    drop_graph(b);
    return build(b);
}

}  // extern "C"
