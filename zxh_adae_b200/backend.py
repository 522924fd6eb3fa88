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

import time
import uuid
from collections.abc import Iterable

from . import _core
from .loader import FRONTEND_GATES, NATIVE_GATES, load_circuit, load_circuit_transpiled


class JobError(RuntimeError):
    """A job that cannot run (qiskit.providers.JobError in the reference)."""


class ExperimentResult:
    """Outcome of one circuit: counts keyed by bitstrings, qubit n-1 first."""

    def __init__(self, counts: dict, sample_time: float, *, shots: int, seed) -> None:
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


class _SimulatorSlot:
    """The one simulator a backend keeps between circuits. It is created at the
    width of the first circuit; a circuit of another width is refused, because
    the simulator's width is fixed at creation (the reference backend keeps one
    cached instance the same way, qiskit_backend.py:256-271)."""

    def __init__(self, factory) -> None:
        self._factory = factory
        self.sim = None

    def for_width(self, num_qubits: int):
        if self.sim is None:
            self.sim = self._factory(num_qubits)
        elif self.sim.num_qubits() != num_qubits:
            raise JobError("ZXH backend caches a single simulator instance. "
                           f"Expected num_qubits={self.sim.num_qubits()}, got num_qubits={num_qubits}.")
        return self.sim

    def release(self) -> None:
        if self.sim is not None:
            self.sim.close()
        self.sim = None


def _reseed(sim, seed) -> None:
    # no seed: the draw stream is whatever the simulator takes without one
    if seed is None:
        sim.clear_seed()
    else:
        sim.set_seed(int(seed))


class Job:
    """Runs its circuits when submitted (the reference's job does the same,
    qiskit_backend.py:150-214); result() afterwards."""

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

    def status(self) -> str:
        return "INITIALIZING" if self._result is None else "DONE"

    def submit(self) -> None:
        if self._result is not None:
            raise JobError("Job already submitted")
        opts = self._options
        shots, seed = int(opts.get("shots", 1)), opts.get("seed_simulator")
        experiments = [
            ExperimentResult(*self._backend._run_circuit(c, shots=shots, seed_simulator=seed,
                                                         optimize_level=opts.get("optimize_level")),
                             shots=shots, seed=seed)
            for c in self._circuits
        ]
        self._result = Result(self._backend.name, self._job_id, experiments)

    def result(self) -> Result:
        if self._result is None:
            raise JobError("Job not submitted")
        return self._result


class Backend:
    """The ``zxh`` backend: ``run(circuits, shots=..., seed_simulator=...)``."""

    name = "zxh"
    description = "ZXH backend (B200)"
    # simulator construction parameters; run() must not be given them
    _BUILD_ONLY = ("disable_x", "eager_expand_all")

    def __init__(self, *, disable_x: bool = False, eager_expand_all: bool = False, dtype: str = "complex128",
                 device: int = 0) -> None:
        self._build = {"disable_x": disable_x, "eager_expand_all": eager_expand_all, "dtype": dtype,
                       "device": device}
        self._slot = _SimulatorSlot(self._make_sim)
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
        return _core.ZXH(num_qubits, **self._build)

    def _run_circuit(self, circuit, *, shots: int, seed_simulator, optimize_level=None) -> tuple:
        """One circuit on the cached simulator: (counts, seconds spent sampling)."""
        sim = self._slot.for_width(circuit.num_qubits)
        _reseed(sim, seed_simulator)
        sim.clear_gates()
        if optimize_level is None:
            load_circuit_transpiled(sim, circuit)
        else:
            load_circuit(sim, circuit, int(optimize_level))
        sim.execute()
        started = time.perf_counter()
        raw = sim.sample_counts(shots)
        elapsed = time.perf_counter() - started
        return {str(word): int(n) for word, n in raw.items()}, elapsed

    def run(self, run_input, **options) -> Job:
        misplaced = sorted(k for k in self._BUILD_ONLY if k in options)
        if misplaced:
            raise JobError(f"{', '.join(misplaced)} is a backend construction parameter for ZXH, "
                           "not a run() option.")
        job = Job(self, _coerce_circuits(run_input), dict(self.options, **options))
        job.submit()
        return job

    def close(self) -> None:
        self._slot.release()


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
