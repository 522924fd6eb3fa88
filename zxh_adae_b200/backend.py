"""A ``zxh`` backend over this library's simulator, without Qiskit.

Follows the run path of the reference's Qiskit backend
(src/zxh/zxhsim/qiskit_backend.py:150-330 of ZXH-Sim): one simulator cached per
backend (a circuit of another width is an error, :256-271), per circuit the seed
set or cleared, the recorded gates cleared, the circuit loaded, execute(), and
``sample_counts(shots)`` timed as the sample time (:273-297); ``run`` refuses the
construction parameters as run options and takes one circuit or an iterable of
circuits (:299-319); the job runs at submit and its result lists per circuit
the counts, the shots, the seed and the sample time (:150-214).

Circuits are used through the Qiskit ``QuantumCircuit`` interface (``.data``,
``.find_bit``, ``.num_qubits``); Qiskit is not imported. Where Qiskit is
installed, the reference's own ``qiskit_backend.py`` also runs unchanged over
``zxh_adae_b200`` in place of its ``_core`` module; this module is the same path
for callers without it. One addition: the run option ``optimize_level`` (None by
default, the reference's ``run``) loads frontend gates through the host circuit
compiler, the work the reference's transpiler stage ``zxh_post`` does
(qiskit_backend.py:135-147).
"""
from __future__ import annotations

import secrets
import time
import uuid
from collections.abc import Iterable

from . import _core
from .loader import FRONTEND_GATES, NATIVE_GATES, load_circuit, load_circuit_transpiled


class JobError(RuntimeError):
    """A job that cannot run (qiskit.providers.JobError in the reference)."""


class ExperimentResult:
    """Outcome of one circuit: counts keyed by bitstrings, qubit n-1 first."""

    def __init__(self, counts: dict, shots: int, seed, sample_time: float) -> None:
        self.counts = counts
        self.shots = shots
        self.seed = seed
        self.success = True
        self.metadata = {"sample_time": sample_time}


class Result:
    def __init__(self, backend_name: str, job_id: str, results: list) -> None:
        self.backend_name = backend_name
        self.job_id = job_id
        self.success = True
        self.results = results

    def get_counts(self, experiment: int | None = None):
        """Counts of one circuit, or of every circuit when the job had several
        and no index is given (the shape of qiskit.result.Result.get_counts)."""
        if experiment is not None:
            return self.results[experiment].counts
        if len(self.results) == 1:
            return self.results[0].counts
        return [r.counts for r in self.results]


class Job:
    def __init__(self, backend: "Backend", circuits: list, options: dict) -> None:
        self._backend = backend
        self._circuits = circuits
        self._options = options
        self._result: Result | None = None
        self._job_id = str(uuid.uuid4())

    def job_id(self) -> str:
        return self._job_id

    def backend(self) -> "Backend":
        return self._backend

    def submit(self) -> None:
        if self._result is not None:
            raise JobError("Job already submitted")
        self._result = self._run_job()

    def status(self) -> str:
        return "DONE" if self._result is not None else "INITIALIZING"

    def result(self) -> Result:
        if self._result is None:
            raise JobError("Job not submitted")
        return self._result

    def _run_job(self) -> Result:
        shots = int(self._options.get("shots", 1))
        seed = self._options.get("seed_simulator")
        level = self._options.get("optimize_level")
        results = []
        for circuit in self._circuits:
            counts, sample_time = self._backend._run_circuit(circuit, shots=shots, seed_simulator=seed,
                                                             optimize_level=level)
            results.append(ExperimentResult(counts, shots, seed, sample_time))
        return Result(self._backend.name, self._job_id, results)


class Backend:
    """The ``zxh`` backend: ``run(circuits, shots=..., seed_simulator=...)``."""

    name = "zxh"
    description = "ZXH backend (B200)"

    def __init__(self, *, disable_x: bool = False, eager_expand_all: bool = False, dtype: str = "complex128",
                 device: int = 0) -> None:
        self._disable_x = disable_x
        self._eager_expand_all = eager_expand_all
        self._dtype = dtype
        self._device = device
        self._sim = None
        self.options = {"shots": 1, "seed_simulator": None, "optimize_level": None}

    @property
    def max_circuits(self) -> None:
        return None

    @property
    def operation_names(self) -> list:
        return sorted(NATIVE_GATES)

    @property
    def frontend_operation_names(self) -> list:
        """Gates accepted with the run option optimize_level set."""
        return sorted(FRONTEND_GATES)

    def _make_sim(self, num_qubits: int):
        return _core.ZXH(num_qubits, disable_x=self._disable_x, eager_expand_all=self._eager_expand_all,
                         dtype=self._dtype, device=self._device)

    def _get_or_create_sim(self, num_qubits: int):
        if self._sim is None:
            self._sim = self._make_sim(num_qubits)
            return self._sim
        if self._sim.num_qubits() != num_qubits:
            raise JobError("ZXH backend caches a single simulator instance. "
                           f"Expected num_qubits={self._sim.num_qubits()}, got num_qubits={num_qubits}.")
        return self._sim

    def _run_circuit(self, circuit, *, shots: int, seed_simulator, optimize_level=None) -> tuple:
        sim = self._get_or_create_sim(circuit.num_qubits)
        if seed_simulator is None:
            clear_seed = getattr(sim, "clear_seed", None)
            if clear_seed is not None:
                clear_seed()
            else:
                sim.set_seed(secrets.randbits(64))
        else:
            sim.set_seed(int(seed_simulator))
        sim.clear_gates()
        if optimize_level is None:
            load_circuit_transpiled(sim, circuit)
        else:
            load_circuit(sim, circuit, int(optimize_level))
        sim.execute()
        t0 = time.perf_counter()
        counts = {str(k): int(v) for k, v in sim.sample_counts(shots).items()}
        return counts, time.perf_counter() - t0

    def run(self, run_input, **options) -> Job:
        invalid = {"disable_x", "eager_expand_all"} & set(options)
        if invalid:
            raise JobError(f"{', '.join(sorted(invalid))} is a backend construction parameter for ZXH, "
                           "not a run() option.")
        job = Job(self, _coerce_circuits(run_input), {**self.options, **options})
        job.submit()
        return job

    def close(self) -> None:
        if self._sim is not None and hasattr(self._sim, "close"):
            self._sim.close()
        self._sim = None


def _is_circuit(obj) -> bool:
    return hasattr(obj, "data") and hasattr(obj, "num_qubits") and hasattr(obj, "find_bit")


def _coerce_circuits(run_input) -> list:
    if _is_circuit(run_input):
        return [run_input]
    if isinstance(run_input, Iterable):
        circuits = list(run_input)
        if all(_is_circuit(c) for c in circuits):
            return circuits
    raise TypeError(f"Unsupported run_input type for ZXH backend: {type(run_input)!r}")


def make_zxh_backend(*, disable_x: bool = False, eager_expand_all: bool = False, **kwargs) -> Backend:
    """make_zxh_backend (src/zxh/zxhsim/__init__.py:46-56); kwargs: dtype, device."""
    return Backend(disable_x=disable_x, eager_expand_all=eager_expand_all, **kwargs)
