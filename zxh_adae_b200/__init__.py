"""B200-native ZXH-Sim state-vector path.

Drop-in for the reference's ``zxhsim`` package entry points on the single-GPU
path (src/zxh/zxhsim/__init__.py of ZXH-Sim): ``ZXH``, ``init``, ``finalize``,
``active``, ``rank``, ``nprocs``, ``PrintRes``, ``load_circuit`` (with the host
circuit compiler, ``optimize_records``), ``load_circuit_transpiled`` and
``make_zxh_backend`` (the ``zxh`` backend's run path without Qiskit).
"""
from __future__ import annotations

from . import _core
from ._core import (
    ZXH,
    PrintRes,
    active,
    as_records,
    finalize,
    init,
    library_path,
    nprocs,
    optimize_records,
    rank,
    version,
)
from .backend import make_zxh_backend
from .loader import compile_circuit, load_circuit, load_circuit_transpiled

__version__ = _core.__version__

__all__ = [
    "ZXH",
    "PrintRes",
    "init",
    "finalize",
    "active",
    "rank",
    "nprocs",
    "as_records",
    "library_path",
    "version",
    "load_circuit_transpiled",
    "load_circuit",
    "compile_circuit",
    "optimize_records",
    "make_zxh_backend",
]
