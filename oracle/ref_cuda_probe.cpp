// ref_cuda_probe.cpp -- test infrastructure only, linked into oracle/_ref/libzxhref_cuda.so
// beside ref_capi.cpp: device-side access to the state of the UNMODIFIED reference CUDA
// backend, so that tests and the benchmark can compare it with this library's state on
// the GPU at 26-30 qubits, where the reference's get_state() (a per-amplitude host
// conversion, src/zxh/src/core/zxh.cpp:579-636) would take minutes.
//
// The reference keeps its state in a private implementation object: class ZXH holds
// `val_t global_phase` and then `std::unique_ptr<impl_t> impl_`
// (src/zxh/include/zxhsim/zxh.h:49-51), and impl_t starts with `size_t N` followed by
// `sv_t sv` (src/zxh/src/core/zxh.cpp:197-198). sv_t's raw_data() and used_bits() are
// public (src/zxh/include/zxhsim/sv.h:25,32). The probe follows that layout and then
// checks what it found: N must equal num_qubits(), the live bits must not exceed
// required_M(), and the buffer must be device memory. Any mismatch returns an error
// and the caller skips the comparison.
#include "zxhsim/sv.h"
#include "zxhsim/zxh.h"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

using namespace ZXHSim;

extern "C" {

// data: device pointer to the real-address state (2^m_bits complex128 amplitudes);
// global phase as (re, im). Returns 0, or 1 when the layout checks fail.
int zxhref_device_state(void *h, const void **data, size_t *m_bits, double *phase_re, double *phase_im)
{
    ZXH &s = *static_cast<ZXH *>(h);
    const unsigned char *obj = reinterpret_cast<const unsigned char *>(h);
    const val_t phase = *reinterpret_cast<const val_t *>(obj);
    const unsigned char *impl = *reinterpret_cast<const unsigned char *const *>(obj + sizeof(val_t));
    if (!impl) return 1;
    const size_t n = *reinterpret_cast<const size_t *>(impl);
    constexpr size_t sv_off = (sizeof(size_t) + alignof(sv_t) - 1) / alignof(sv_t) * alignof(sv_t);
    const sv_t &sv = *reinterpret_cast<const sv_t *>(impl + sv_off);
    if (n != s.num_qubits()) return 1;
    const size_t m = sv.used_bits();
    if (m > s.required_M()) return 1;
    const val_t *p = sv.raw_data();
    cudaPointerAttributes attr{};
    if (!p || cudaPointerGetAttributes(&attr, p) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return 1;
    }
    *data = p;
    *m_bits = m;
    *phase_re = phase.real();
    *phase_im = phase.imag();
    return 0;
}

// Waits for the device (the reference launches on the legacy default stream).
int zxhref_device_sync(void)
{
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

} // extern "C"
