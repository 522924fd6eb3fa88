"""Test and measurement infrastructure only: compares two device-resident states.

Used by the GPU parity tests and by bench.py's baseline legs to compare this
library's state with the reference CUDA backend's (``Reference.device_state``) or
with another run of this library, without copying 2^30 amplitudes to the host.
Both states are given as raw device pointers (real-address order, complex64 or
complex128) with their global phases; the comparison runs on the GPU in FP64,
in chunks, so it needs at most a few hundred MiB of extra device memory.
"""
from __future__ import annotations

import torch


class _CudaArray:
    def __init__(self, ptr: int, count: int, typestr: str) -> None:
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def device_view(ptr: int, m_bits: int, elem_bytes: int, device: int = 0) -> torch.Tensor:
    """A torch view (no copy) of 2^m_bits amplitudes at a device pointer."""
    ts = {8: "<c8", 16: "<c16"}[elem_bytes]
    return torch.as_tensor(_CudaArray(ptr, 1 << m_bits, ts), device=f"cuda:{device}")


def compare(a: torch.Tensor, phase_a: complex, b: torch.Tensor, phase_b: complex, chunk: int = 1 << 25) -> dict:
    """max |phase_a a - phase_b b| and the fidelity error 1 - |<a|b>|^2 / (<a|a><b|b>),
    both in FP64 on the device (the global phases scale every amplitude)."""
    if a.numel() != b.numel():
        raise ValueError(f"state sizes differ: {a.numel()} vs {b.numel()}")
    pa = torch.tensor(phase_a, dtype=torch.complex128, device=a.device)
    pb = torch.tensor(phase_b, dtype=torch.complex128, device=b.device)
    mx = torch.zeros((), dtype=torch.float64, device=a.device)
    dot = torch.zeros((), dtype=torch.complex128, device=a.device)
    na = torch.zeros((), dtype=torch.float64, device=a.device)
    nb = torch.zeros((), dtype=torch.float64, device=a.device)
    for i in range(0, a.numel(), chunk):
        x = a[i:i + chunk].to(torch.complex128) * pa
        y = b[i:i + chunk].to(torch.complex128) * pb
        mx = torch.maximum(mx, (x - y).abs().max())
        dot += torch.vdot(y, x)
        na += (x.abs() ** 2).sum()
        nb += (y.abs() ** 2).sum()
    fid = 1.0 - abs(complex(dot)) ** 2 / (float(na) * float(nb))
    return {"max_abs": float(mx), "fidelity_err": float(fid), "norm_a": float(na), "norm_b": float(nb)}
