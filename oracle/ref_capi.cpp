// ref_capi.cpp -- test infrastructure only: a C ABI over the UNMODIFIED reference
// ZXH-Sim core (AxEquals-b/ZXH_ADAE, src/zxh), compiled from the reference's own
// sources by oracle/Makefile into oracle/_ref/. Nothing in the product links this.
//
// It wraps the public C++ API of src/zxh/include/zxhsim/zxh.h:11-53 the way the
// reference's pybind11 module does (src/zxh/src/pybind/bindings.cpp:79-118), so a
// ctypes caller can drive the reference exactly as _core.ZXH would.
#include "zxhsim/runtime.h"
#include "zxhsim/zxh.h"

#include <cstdint>
#include <cstring>
#include <vector>

using namespace ZXHSim;

namespace
{
struct rec_t
{
    uint32_t type;
    uint32_t cq;
    uint32_t q;
    uint32_t reserved;
    double theta;
    double lambda;
    double phi;
};

void ensure_init()
{
    if (!active())
        init(nullptr, nullptr);
}
} // namespace

extern "C" {

void *zxhref_create(size_t n, int disable_x, int eager_expand_all)
{
    ensure_init();
    return new ZXH(n, disable_x != 0, eager_expand_all != 0);
}

void zxhref_destroy(void *h)
{
    delete static_cast<ZXH *>(h);
}

// Records gates through the per-gate methods (zxh.cpp:234-310). Gate codes follow
// gate_type_t (defs.h:61-74); 11 = Rx.
int zxhref_push(void *h, const void *recs, size_t count)
{
    ZXH &s = *static_cast<ZXH *>(h);
    const rec_t *g = static_cast<const rec_t *>(recs);
    for (size_t i = 0; i < count; i++)
    {
        switch (g[i].type)
        {
        case 1: s.Barrier(); break;
        case 2: s.Z(g[i].q); break;
        case 3: s.Rz(g[i].q, g[i].theta); break;
        case 4: s.P(g[i].q, g[i].theta); break;
        case 5: s.CRz(g[i].cq, g[i].q, g[i].theta); break;
        case 6: s.CP(g[i].cq, g[i].q, g[i].theta); break;
        case 7: s.X(g[i].q); break;
        case 8: s.CX(g[i].cq, g[i].q); break;
        case 9: s.H(g[i].q); break;
        case 10: s.U3(g[i].q, g[i].theta, g[i].lambda, g[i].phi); break;
        case 11: s.Rx(g[i].q, g[i].theta); break;
        default: return 1;
        }
    }
    return 0;
}

void zxhref_execute(void *h)
{
    static_cast<ZXH *>(h)->execute();
}

size_t zxhref_required_M(void *h)
{
    return static_cast<ZXH *>(h)->required_M();
}

// get_state() (zxh.cpp:579-636): 2^n complex128, interleaved re/im.
void zxhref_get_state(void *h, double *out)
{
    const std::vector<val_t> st = static_cast<ZXH *>(h)->get_state();
    std::memcpy(out, st.data(), st.size() * sizeof(val_t));
}

// set_seed + measure alone (zxh.cpp:216-220,555-559): the draw, for timing.
void zxhref_measure(void *h, uint64_t seed, size_t shots)
{
    ZXH &s = *static_cast<ZXH *>(h);
    s.set_seed(seed);
    s.measure(shots);
}

// set_seed + measure + get_results (zxh.cpp:216-220,555-564); packs each result
// into ceil(n/64) words, bit q = virtual qubit q.
void zxhref_sample(void *h, uint64_t seed, size_t shots, uint64_t *words)
{
    ZXH &s = *static_cast<ZXH *>(h);
    s.set_seed(seed);
    s.measure(shots);
    const size_t n = s.num_qubits();
    std::vector<res_t> res(shots, res_t(n, false));
    s.get_results(res.data(), shots);
    const size_t wc = (n + 63) / 64;
    std::memset(words, 0, shots * wc * sizeof(uint64_t));
    for (size_t i = 0; i < shots; i++)
        for (size_t q = 0; q < n; q++)
            if (res[i].get_bit(q))
                words[i * wc + (q >> 6)] |= (uint64_t(1) << (q & 63));
}

} // extern "C"
