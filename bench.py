"""Benchmark of the B200-native ZXH path (one JSON line on stdout, rank 0).

Default workload (configuration 2, the diagonal-batch microbenchmark): a
30-qubit complex64 state (8 GiB) prepared with H on every qubit; one step applies
one batch of B = 4096 seeded random p/cp gates (50/50, angles uniform [0, 2 pi))
as one read-modify-write pass of the state. The state (8 GiB) is larger than L2
(126 MB), so no flush is needed between steps.

* value        whole-job GB/s from the device time of the pass kernels
               (algorithmic bytes 2 * 2^30 * 8 per pass), inputs resident.
* e2e          the same metric through the C ABI with host gate records, timed on
               the host around K zxh_apply_async calls and the closing zxh_sync
               (every step: host planning, program upload from pinned memory,
               launch, status read-back; the next step is planned while the GPU
               runs the current one); sync_api_value: the same through the
               blocking zxh_apply.
* roofline     the dominant kernel against the measured HBM copy bandwidth in
               MEASURED_PEAKS.json; traffic = its DRAM bytes per launch from the
               committed ncu summary under profiles/.
* cpu_baseline the reference ZXH-Sim OpenMP backend (compiled from its own sources
               into oracle/_ref) on a bounded sample: the same B = 4096 batch
               distribution on an 18-qubit complex128 state, timed with the
               reference's header-subtraction method, GB/s at 16 B/amplitude.
* config2      configuration 2 in full: B in {64, 256, 1024, 4096} random p/cp and
               the 435-pair cp cascade at 30 qubits, complex64 and complex128:
               gates/s, passes/s, GB/s, fraction of the HBM peak, the complex64
               fidelity error against complex128.
* u3_layer     the U3-batch half of the 30-qubit target: one layer of U3 on every
               qubit of the same complex64 state, its passes and GB/s per pass
               (u3_layer_c128: the same in complex128).
* sampler      10^6 shots from the 30-qubit state (sampler_c128: complex128).
* config1      configuration 1 (20 qubits, complex128 and complex64, 1024 shots).
* config3      configuration 3 (32 qubits complex64: 40 x [U3 all; cz matching],
               4 layers against complex128, the hidden-string circuit, 10^6 shots).
* batch        configuration 5: energies and adjoint gradients of 512 uneven
               circuits, every pass as its own launch vs one persistent launch vs
               its CUDA-graph replay (autotuned), and the plain per-circuit API.
* adjoint      the second half of the metric, on the 24-qubit, 432-parameter
               hardware-efficient ansatz (8 x [RY, RZ on every qubit; CX chain] +
               final RY/RZ, parameters uniform [-pi, pi)) with the TFIM observable
               sum Z_i Z_{i+1} + sum X_i: gradients/s of one adjoint sweep
               (complex64 state, FP64 reductions, checkpoint every 48 parameters)
               against gradients/s of parameter shift (864 energies on the plain
               forward path, complex64), both timed on the host through the public
               API and as summed kernel time, and the max |error| of both against
               FP64 central differences (step 1e-6) on the complex128 forward path.
* gpu_baseline the reference's own GPU path (its CUDA backend compiled for sm_100a
               from its sources) timed on the same GPU on configuration 2's
               batches, one U3 layer and 10^6 shots at 30 qubits (complex128, the
               reference's header-subtraction method), beside this library's times
               for the same work, and the two complex128 states compared on the
               device. Like cpu_baseline it is a baseline leg: it runs the
               reference, never this library's path through the oracle.
Rank 0 at N = 1 only, for every leg after the headline.

``--workload u3|adjoint|batch|sample|config2|config3`` time those legs alone (the
commands the ncu summaries under profiles/ were taken with). ``--impl reference``
runs the reference CPU backend alone and prints its line; that process imports
the workload generators without loading this library. Multi-GPU (``torchrun``):
the path does not shard, each rank runs an independent replica; value is the sum
over ranks, times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "30q GB/s vs HBM peak; adjoint vs param-shift grads/s at <=1e-5 err, 1 GPU"
UNIT = "GB/s"
N_QUBITS = 30
BATCH = 4096
REF_SAMPLE_QUBITS = 18


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)  # ~0.3 s timed: several clock samples land inside
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="diag",
                    choices=["diag", "cxwindow", "u3", "adjoint", "batch", "sample", "config2", "config3"])
    ap.add_argument("--dtype", default="complex64", choices=["complex64", "complex128"],
                    help="diag / cxwindow / u3 workloads: the state's type")
    ap.add_argument("--set-param", action="append", default=[], metavar="NAME=VALUE",
                    help="planner knob (zxh_set_param) on the headline workload's simulators, e.g. span=0")
    ap.add_argument("--no-tune", action="store_true", help="batch workload: skip the autotuner")
    ap.add_argument("--batch-count", type=int, default=512, help="batch workload: circuits")
    ap.add_argument("--no-extras", action="store_true", help="skip the U3-layer and adjoint legs of the diag line")
    ap.add_argument("--no-adjoint-checks", action="store_true", help="adjoint workload: skip parameter shift and FD")
    ap.add_argument("--no-gpu-baseline", action="store_true", help="skip timing the reference CUDA backend")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float, local: int) -> float:
    if pg is None:
        return x
    import torch

    # local < 0: CPU tensor (gloo process groups, as in the CPU tests)
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}" if local >= 0 else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """Samples SM clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"zxh_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is up (its first line written)
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 2.0 and self.path.stat().st_size == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name: str):
    """DRAM bytes per launch of a kernel from a committed ncu summary, if any."""
    p = ROOT / "profiles" / name
    if not p.is_file():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch"):
            try:
                return float(line.split("=")[1].split()[0])
            except Exception:
                return None
    return None


# --------------------------------------------------------------------------- reference CPU


def standalone_workloads():
    """zxh_adae_b200.workloads and the pure-numpy records module it uses, imported
    without running the package's __init__ (which loads libzxhb200.so): the
    reference arm generates the same gate lists but must not load this library.
    Where the package is already imported, that module is returned."""
    import importlib
    import types

    name = "zxh_adae_b200"
    if name in sys.modules:
        return importlib.import_module(name + ".workloads")
    stub = types.ModuleType(name)
    stub.__path__ = [str(ROOT / name)]
    sys.modules[name] = stub
    try:
        return importlib.import_module(name + ".workloads")
    finally:
        del sys.modules[name]  # a later `import zxh_adae_b200` runs the real package


def ref_cpu_sample(steps: int, warmup: int, batch: int):
    """Reference OpenMP backend, diag batch on a REF_SAMPLE_QUBITS-qubit state,
    header-subtracted as the reference's diag microbenchmark does
    (benchmarks/runners/diag_batch_microbench.py:209-231), 16 B/amplitude."""
    from oracle.bridge import Reference, ref_available

    wl = standalone_workloads()

    if not ref_available("omp"):
        return None
    n = REF_SAMPLE_QUBITS
    header = wl.h_all(n)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    os.environ["OMP_NUM_THREADS"] = str(cores)
    bytes_step = 2 * (1 << n) * 16
    times = []
    for k in range(warmup + steps):
        full = np.concatenate([header, wl.diag_batch(n, batch, seed=1000 + k)])
        hs = Reference(n, backend="omp")
        hs.push(header)
        fs = Reference(n, backend="omp")
        fs.push(full)

        def ex(sim):
            t0 = time.perf_counter()
            sim.execute()
            return time.perf_counter() - t0

        h1 = ex(hs)
        f1 = ex(fs)
        f2 = ex(fs)
        h2 = ex(hs)
        d = max(1e-9, 0.5 * ((f1 - h1) + (f2 - h2)))
        if k >= warmup:
            times.append(d)
    t = sum(times) / len(times)
    return {
        "value": bytes_step / t / 1e9,
        "unit": UNIT,
        "cores": cores,
        "kind": "reference",
        "sample": f"reference omp backend, {n}-qubit complex128 state, H header + B={batch} random p/cp "
                  f"(50/50), header-subtracted execute(), mean of {len(times)} steps "
                  f"({1e3 * t:.1f} ms/step), GB/s at 2*2^{n}*16 B",
        "ms_per_step": 1e3 * t,
    }


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    if rank != 0:
        return
    # a step is about 0.3 s on 16 host cores: the requested warm-up (at most 10) and
    # up to 30 timed steps keep the run within a minute
    steps, warmup = min(args.steps, 30), min(args.warmup, 10)
    cb = ref_cpu_sample(steps, warmup, args.batch)
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference OpenMP backend not built (oracle/_ref)"}))
        return
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": cb["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128",
        "data": "synthetic",
        "config": {"workload": f"diag-batch {REF_SAMPLE_QUBITS}q complex128 B={args.batch} random p/cp "
                               "(bounded CPU sample of the 30q workload)",
                   "qubits": REF_SAMPLE_QUBITS, "batch": args.batch},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# --------------------------------------------------------------------------- ours


def adjoint_leg(local: int, n: int = 24, reps: int = 8, checkpoint_every: int = 48, steps: int = 5,
                warmup: int = 1, checks: bool = True) -> dict:
    """Adjoint gradients/s vs parameter-shift gradients/s on the same GPU."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import adjoint as ad

    circ = ad.hardware_efficient_ansatz(n, reps)
    terms = ad.tfim_terms(n)
    p = np.random.default_rng(2024).uniform(-np.pi, np.pi, circ.nparams)
    s64 = zx.ZXH(n, dtype="complex64", device=local)
    for _ in range(max(warmup, 1)):
        ad.adjoint(s64, circ, p, terms, checkpoint_every)
    dev = []
    t0 = time.perf_counter()
    for _ in range(steps):
        e, g = ad.adjoint(s64, circ, p, terms, checkpoint_every)
        dev.append(s64.last_stats()[2])
    t_adj = (time.perf_counter() - t0) / steps
    kernels = s64.last_stats()[0]
    d = {
        "workload": f"{n}q complex64 hardware-efficient ansatz L={reps} (RY, RZ all + CX chain, final RY/RZ), "
                    f"{circ.nparams} params, TFIM sum ZZ + 1.0 sum X (open)",
        "params": circ.nparams,
        "adjoint_ms": 1e3 * t_adj,
        "adjoint_device_ms": statistics.mean(dev),
        "adjoint_kernels": kernels,
        "adjoint_grads_per_s": circ.nparams / t_adj,
        "energy": e,
        "checkpoint_every": checkpoint_every,
    }
    if checks:
        ad.energy(s64, circ, p, terms)  # warm-up of the forward path
        ps_dev = []
        t0 = time.perf_counter()
        g_ps = ad.parameter_shift(s64, circ, p, terms, device_ms=ps_dev)
        t_ps = time.perf_counter() - t0
        s128 = zx.ZXH(n, dtype="complex128", device=local)
        e128 = ad.energy(s128, circ, p, terms)
        fd = ad.finite_difference(s128, circ, p, terms, 1e-6)
        s128.close()
        d.update({
            "param_shift_s": t_ps,
            "param_shift_grads_per_s": circ.nparams / t_ps,
            "speedup": t_ps / t_adj,
            # kernel time only (execute + expectation of each of the 864 energies vs
            # the adjoint call's kernels): the share of the speed-up that is not host work
            "param_shift_energies": len(ps_dev),
            "param_shift_device_s": sum(ps_dev) / 1e3,
            "speedup_device": (sum(ps_dev) / 1e3) / (statistics.mean(dev) / 1e3),
            "energy_err_vs_c128": abs(e - e128),
            "max_abs_err_vs_fp64_fd": float(np.max(np.abs(g - fd))),
            "param_shift_max_abs_err_vs_fp64_fd": float(np.max(np.abs(g_ps - fd))),
            "fd": "central differences, step 1e-6, complex128 forward path",
        })
    s64.close()
    return d


def batch_leg(local: int, count: int = 512, seed: int = 2025, tune: bool = True, api: bool = True) -> dict:
    """Configuration 5: 512 circuits (n uniform in {10..22}, 20 layers of U3 on every
    qubit + cp chain, own TFIM each) -> energies and adjoint gradients of all of
    them, complex64: every pass as its own launch vs one persistent launch vs its
    CUDA-graph replay (after the autotuner), device time (CUDA events)."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl
    from zxh_adae_b200.batch import Batch

    circ = wl.batch_tfim(count, seed)
    t0 = time.perf_counter()
    b = Batch([(c[0], c[1], c[2]) for c in circ], dtype="complex64", device=local)
    create_s = time.perf_counter() - t0
    tuned = b.tune(1) if tune else None
    ops, tasks, _ = b.stats()
    d = {"workload": f"{count} circuits, n uniform in 10..22, 20 x [U3 all; cp chain], TFIM h in [0.5, 1.5], "
                     "energy + adjoint gradient of every circuit, complex64",
         "circuits": count, "amplitudes": int(sum(1 << c[0] for c in circ)),
         "gradients": int(b.grad_offsets[-1]), "ops": ops, "tasks": tasks, "create_s": create_s, "tuned": tuned}
    res = {}
    for mode in ("sequential", "persistent", "graph"):
        b.run(mode)
        best = 1e300
        for _ in range(2):
            e, g = b.run(mode)
            best = min(best, b.stats()[2])
        res[mode] = (best, e, g)
        d[f"{mode}_ms"] = best
    d["state_bytes_per_run"] = b.state_bytes()
    peak, kind = peaks()
    for mode in ("sequential", "persistent", "graph"):
        d[f"{mode}_GBps"] = d["state_bytes_per_run"] / (d[f"{mode}_ms"] / 1e3) / 1e9
    d["graph_frac_of_peak"] = d["graph_GBps"] / peak
    d["speedup_persistent_vs_sequential"] = d["sequential_ms"] / d["persistent_ms"]
    d["speedup_graph_vs_sequential"] = d["sequential_ms"] / d["graph_ms"]
    d["max_grad_diff_modes"] = float(max(np.max(np.abs(res[m][2] - res["sequential"][2])) for m in res))
    # every result against complex128: the same batch in complex128
    e64, g64 = res["graph"][1], res["graph"][2]
    b.close()
    b128 = Batch([(c[0], c[1], c[2]) for c in circ], dtype="complex128", device=local)
    e128, g128 = b128.run("persistent")
    b128.close()
    d["energy_max_err_vs_complex128"] = float(np.max(np.abs(e64 - e128)))
    d["grad_max_err_vs_complex128"] = float(np.max(np.abs(g64 - g128)))
    if api:  # the plain per-circuit API, one circuit after another (host planning included)
        sims = {}
        t0 = time.perf_counter()
        for n, rec, terms, _h in circ:
            s = sims.get(n) or sims.setdefault(n, zx.ZXH(n, dtype="complex64", device=local))
            s.clear_gates()
            s.push_gates(rec)
            s.adjoint_gradient(terms)
        d["api_per_circuit_ms"] = 1e3 * (time.perf_counter() - t0)
        for s in sims.values():
            s.close()
    return d


def _device_state(ptr: int, m: int, eb: int):
    import torch

    class _CAI:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (1 << m,), "typestr": "<c8" if eb == 8 else "<c16",
                                             "data": (ptr, False), "version": 3}

    return torch.as_tensor(_CAI(), device="cuda")


def compare_states(a, phase_a: complex, b, phase_b: complex) -> dict:
    """max |phase_a a - phase_b b| and 1 - |<a|b>|^2 / (<a|a><b|b>) of two device
    states (torch views, real-address order), in FP64 on the device, chunked."""
    import torch

    if a.numel() != b.numel():
        return {"max_abs": float("nan"), "fidelity_err": float("nan")}
    pa = torch.tensor(phase_a, dtype=torch.complex128, device="cuda")
    pb = torch.tensor(phase_b, dtype=torch.complex128, device="cuda")
    mx = torch.zeros((), dtype=torch.float64, device="cuda")
    acc = torch.zeros((), dtype=torch.complex128, device="cuda")
    na = torch.zeros((), dtype=torch.float64, device="cuda")
    nb = torch.zeros((), dtype=torch.float64, device="cuda")
    step = 1 << 26
    for i in range(0, a.numel(), step):
        x = a[i:i + step].to(torch.complex128) * pa
        y = b[i:i + step].to(torch.complex128) * pb
        mx = torch.maximum(mx, (x - y).abs().max())
        acc += torch.vdot(y, x)
        na += (x.abs() ** 2).sum()
        nb += (y.abs() ** 2).sum()
    return {"max_abs": float(mx), "fidelity_err": float(1.0 - abs(complex(acc)) ** 2 / (float(na) * float(nb)))}


def fidelity_err(sim_a, sim_b) -> float:
    """1 - |<a|b>|^2 / (<a|a><b|b>) of two simulators' states (same map and size)."""
    pa, ma, ea, ga = sim_a.state_view()
    pb, mb, eb, gb = sim_b.state_view()
    if ma != mb:
        return float("nan")
    return compare_states(_device_state(pa, ma, ea), ga, _device_state(pb, mb, eb), gb)["fidelity_err"]


CONFIG2_BATCHES = (64, 256, 1024, 4096)
CX_CHAIN_BATCHES = (256, 4096)  # the same windows after a CX chain (multi-bit selectors)


def config2_leg(local: int, n: int = N_QUBITS, steps: int = 5, warmup: int = 2) -> dict:
    """Configuration 2 at n qubits: an H-prepared state, then per step one batch of
    B random p/cp gates (B in 64, 256, 1024, 4096; 50/50, angles uniform [0, 2 pi))
    or the full controlled-phase cascade (every pair j > i, angle pi / 2^(j - i)), in
    complex64 and complex128. Per batch: device ms (CUDA events on the library's
    stream), ms through the blocking API (host planning included), gates/s,
    passes/s, GB/s at 2 x state bytes per pass and the fraction of the measured HBM
    peak; then the fidelity error of the complex64 state against the complex128
    one after all the same batches."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    peak, kind = peaks()
    keys = list(CONFIG2_BATCHES) + ["cascade"] + [f"cx_chain+{B}" for B in CX_CHAIN_BATCHES]
    batches = {B: [wl.diag_batch(n, B, seed=7000 + 10 * B + k) for k in range(warmup + steps)]
               for B in CONFIG2_BATCHES}
    batches["cascade"] = [wl.cp_cascade(n)] * (warmup + steps)
    for B in CX_CHAIN_BATCHES:
        batches[f"cx_chain+{B}"] = [wl.diag_batch(n, B, seed=8000 + 10 * B + k) for k in range(warmup + steps)]
    rows = {k: {"batch": k, "gates": int(len(batches[k][0]))} for k in keys}
    sims = {}
    for dtype, eb in (("complex64", 8), ("complex128", 16)):
        sim = zx.ZXH(n, dtype=dtype, device=local)
        sim.push_gates(wl.h_all(n))
        sim.execute()
        chained = False
        for k in keys:
            if str(k).startswith("cx_chain") and not chained:
                # CX(i, i+1) chain: map updates only; every later selector is a
                # parity of several real bits (the Walsh-sum window pass)
                sim.apply(wl.cx_chain(n))
                chained = True
            dev_ms, launches, passes, wall, _ = timed_applies(sim, batches[k], warmup, steps, None, local)
            ms = sum(dev_ms) / steps
            pps = passes / steps
            gbps = pps * 2 * (1 << n) * eb / (ms / 1e3) / 1e9
            rows[k]["c64" if eb == 8 else "c128"] = {
                "ms": ms, "api_ms": 1e3 * wall / steps, "passes": pps, "kernels": launches / steps,
                "gates_per_s": rows[k]["gates"] / (ms / 1e3), "passes_per_s": pps / (ms / 1e3),
                "GBps": gbps, "frac_of_peak": gbps / peak}
        sims[dtype] = sim
    fid = fidelity_err(sims["complex64"], sims["complex128"])
    for s in sims.values():
        s.close()
    return {"workload": f"{n}q H-prepared; per step B random p/cp (50/50) or the {n * (n - 1) // 2}-pair cp cascade; "
                        "then a CX chain and B random p/cp (selectors are parities of several real bits)",
            "peak": peak, "peak_kind": kind, "rows": [rows[k] for k in keys],
            "complex64_fidelity_err_vs_complex128": fid, "steps": steps, "warmup": warmup}


def config1_leg(local: int, seed: int = 2024) -> dict:
    """Configuration 1: 20 qubits, complex128, H on all + 10 x [U3 all; cp chain], 1024
    shots; device ms of execute and measure, and the complex64 run's fidelity error."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    g = wl.plain_layers(20, 10, seed)
    out = {"workload": "20q complex128, H all + 10 x [U3 all; cp (i, i+1)], 1024 shots"}
    sims = {}
    for dtype in ("complex128", "complex64"):
        s = zx.ZXH(20, dtype=dtype, device=local)
        s.push_gates(g)
        s.execute()
        s.execute()
        k, p, ms = s.last_stats()
        s.set_seed(seed)
        s.measure(1024)
        out[dtype] = {"execute_ms": ms, "passes": p, "kernels": k, "measure_1024_ms": s.last_stats()[2]}
        sims[dtype] = s
    out["complex64_fidelity_err_vs_complex128"] = fidelity_err(sims["complex64"], sims["complex128"])
    w64, w128 = sims["complex64"].results_words(), sims["complex128"].results_words()
    out["complex64_sample_mismatch_vs_complex128"] = float(np.mean(w64 != w128))
    for s in sims.values():
        s.close()
    return out


def config3_leg(local: int, seed: int = 33) -> dict:
    """Configuration 3: 32 qubits complex64, 40 x [U3 all; cz matching] (4 layers also in
    complex128 for the fidelity error), then the 31+1-qubit hidden-string circuit and
    10^6 shots (every shot must read the secret)."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    n = 32
    out = {"workload": "32q complex64: 40 x [U3 all; cz on a random perfect matching]; hidden string 31+1, 10^6 shots"}
    g4 = wl.u3_matching_layers(n, 4, seed)
    s64 = zx.ZXH(n, dtype="complex64", device=local)
    s64.push_gates(g4)
    s64.execute()
    s128 = zx.ZXH(n, dtype="complex128", device=local)
    s128.push_gates(g4)
    s128.execute()
    out["layers4_fidelity_err_vs_complex128"] = fidelity_err(s64, s128)
    s128.close()
    g40 = wl.u3_matching_layers(n, 40, seed)
    s64.clear_gates()
    s64.push_gates(g40)
    s64.execute()
    k, p, ms = s64.last_stats()
    out["layers40_ms"] = ms
    out["layers40_passes"] = p
    out["layers40_pass_GBps"] = p * 2 * (1 << n) * 8 / (ms / 1e3) / 1e9
    recs, secret = wl.hidden_string(31, seed + 1)
    s64.clear_gates()
    s64.push_gates(recs)
    s64.execute()
    out["hidden_execute_ms"] = s64.last_stats()[2]
    out["hidden_passes"] = s64.last_stats()[1]
    s64.set_seed(99)
    s64.measure(1_000_000)
    out["hidden_measure_1e6_ms"] = s64.last_stats()[2]
    w = s64.results_words()
    data = np.unique(w & np.uint64((1 << 31) - 1))
    out["hidden_all_shots_read_secret"] = bool(len(data) == 1 and int(data[0]) == secret)
    s64.close()
    return out


def sampler_leg(local: int, n: int = N_QUBITS, shots: int = 1_000_000, steps: int = 5,
                dtype: str = "complex64") -> dict:
    """10^6 multinomial shots from an n-qubit state (H on all + one U3 layer);
    roofline = one read of the state (2^n x 8 or 16 B). Device ms (CUDA events)
    and the wall time of the measure call."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    eb = 8 if dtype == "complex64" else 16
    sim = zx.ZXH(n, dtype=dtype, device=local)
    sim.push_gates(np.concatenate([wl.h_all(n), wl.u3_layer(n, seed=5)]))
    sim.execute()
    sim.set_seed(11)
    sim.measure(shots)
    ms, wall = [], []
    for k in range(steps):
        sim.set_seed(100 + k)
        t0 = time.perf_counter()
        sim.measure(shots)
        wall.append(time.perf_counter() - t0)
        ms.append(sim.last_stats()[2])
    kernels = sim.last_stats()[0]
    out = {}
    if dtype == "complex64":
        # counts of the last draw: on the device (zxh_counts: only the distinct
        # outcomes cross to the host) vs every shot copied and np.unique'd on the host
        cw, hw = [], []
        for k in range(3):
            t0 = time.perf_counter()
            words, cnt = sim.counts_words()
            cw.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            hk, hc = np.unique(sim.results_words(), return_counts=True)
            hw.append(time.perf_counter() - t0)
        same = bool(np.array_equal(words, hk) and np.array_equal(cnt, hc.astype(np.uint64)))
        out["counts"] = {"distinct": int(len(words)), "device_counts_wall_ms": min(cw) * 1e3,
                         "host_unique_wall_ms": min(hw) * 1e3, "identical": same}
    sim.close()
    t = statistics.median(ms)
    peak, kind = peaks()
    gbps = (1 << n) * eb / (t / 1e3) / 1e9
    return {"workload": f"{shots} shots from a {n}-qubit {dtype} state (H all + one U3 layer)", "ms": t,
            "api_ms": 1e3 * statistics.median(wall), "shots_per_s": shots / (t / 1e3), "state_read_GBps": gbps,
            "frac_of_peak": gbps / peak, "kernels": kernels, "bytes": "one read of the state", **out}


def timed_applies(sim, batches, warmup, steps, pg, local):
    """W untimed applies, then K timed ones: per-step device ms (CUDA events on the
    library's stream around the pass kernels), launches, passes, host wall time.
    An apply ending with U3 gates leaves their last phases to the next apply's
    first window; the phases the K-th one leaves are applied (flush) inside the
    timed region and counted with the last step."""
    for k in range(warmup):
        sim.apply(batches[k])
    barrier(pg)
    dev_ms, launches, passes = [], 0, 0
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        for k in range(steps):
            sim.apply(batches[warmup + k])
            kk, pp, ms = sim.last_stats()
            dev_ms.append(ms)
            launches += kk
            passes += pp
        sim.flush()
        kk, pp, ms = sim.last_stats()
        if pp:
            dev_ms[-1] += ms
            launches += kk
            passes += pp
        wall = time.perf_counter() - t0
    barrier(pg)
    return dev_ms, launches, passes, wall, clk.summary()


def timed_async(n, dtype, local, batches, warmup, steps, pg, prefix=None, knobs=()) -> float:
    """End-to-end wall time of K zxh_apply_async calls and the closing zxh_sync on a
    fresh H-prepared simulator: every step plans on the host, uploads its program
    from pinned memory and reads its status word back; step k + 1 is planned while
    step k runs on the GPU."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    sim = zx.ZXH(n, dtype=dtype, device=local)
    for k, v in knobs:
        sim.set_param(k, v)
    sim.push_gates(wl.h_all(n))
    sim.execute()
    if prefix is not None:
        sim.apply(prefix)
    for k in range(warmup):
        sim.apply_async(batches[k])
    sim.sync()
    barrier(pg)
    t0 = time.perf_counter()
    for k in range(steps):
        sim.apply_async(batches[warmup + k])
    sim.sync()
    sim.flush()  # phases the last step left over, if any
    wall = time.perf_counter() - t0
    barrier(pg)
    sim.close()
    return wall


def u3_leg(local: int, n: int = N_QUBITS, steps: int = 20, warmup: int = 3, dtype: str = "complex64") -> dict:
    """One U3 layer (U3 on every qubit) per step on the n-qubit state, K = 20 layers
    timed (about 0.2 s complex64, 0.45 s complex128) and the closing flush of the
    last layer's phases counted with them; complex64 also reports its fidelity
    error against the same layers in complex128."""
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    eb = 8 if dtype == "complex64" else 16
    sim = zx.ZXH(n, dtype=dtype, device=local)
    sim.push_gates(wl.h_all(n))
    sim.execute()
    layers = [wl.u3_layer(n, seed=500 + k) for k in range(warmup + steps)]
    dev_ms, launches, passes, wall, _ = timed_applies(sim, layers, warmup, steps, None, local)
    fid = None
    if dtype == "complex64":
        ref = zx.ZXH(n, dtype="complex128", device=local)
        ref.push_gates(np.concatenate([wl.h_all(n)] + layers))
        ref.execute()
        fid = fidelity_err(sim, ref)
        ref.close()
    sim.close()
    state = (1 << n) * eb
    ms = sum(dev_ms) / steps
    gbps = (passes / steps) * 2 * state / (ms / 1e3) / 1e9
    peak, kind = peaks()
    return {"workload": f"U3 on all {n} qubits of a {dtype} state, random angles, one layer per step "
                        "(the phases each layer leaves ride in the next layer's first window; the last "
                        "layer's are applied after the K layers and counted in the time)",
            "ms_per_layer": ms, "api_ms_per_layer": 1e3 * wall / steps, "passes_per_layer": passes / steps,
            "kernels_per_layer": launches / steps, "gates_per_s": n / (ms / 1e3),
            "passes_per_s": (passes / steps) / (ms / 1e3), "pass_GBps": gbps, "frac_of_peak": gbps / peak,
            "layer_GBps": 2 * state / (ms / 1e3) / 1e9, "layer_frac_of_peak": 2 * state / (ms / 1e3) / 1e9 / peak,
            "peak": peak, "peak_kind": kind, "fidelity_err_vs_complex128": fid,
            "bytes": "2 x state per pass (one read and one write)"}


def gpu_baseline_leg(local: int, ours: dict, n: int = N_QUBITS, seed: int = 4242) -> dict:
    """The reference's own GPU path, timed on this GPU: ZXH-Sim's CUDA backend
    (kernel_cuda.cu / measure_cuda.cu, compiled for sm_100a from the reference's
    sources into oracle/_ref; complex128 only) on configuration 2's batches, one
    U3 layer on all n qubits and 10^6 shots, n = 30. Its execute() ends with a
    device synchronize (zxh.cpp:550-551), so each item is timed on the host with
    the reference's header-subtraction method (diag_batch_microbench.py:209-231):
    an H-on-all header run and the header + item run, alternated H F F H, and
    the item's time is the mean of the two differences. Beside each item: this
    library's complex128 and complex64 times for the same work (device and
    through the blocking API, from the legs above) and the ratios. After the
    B = 4096 and U3-layer items, the reference's state and this library's
    complex128 state for the same gate list are compared on the device."""
    from oracle.bridge import Reference, ref_available
    from zxh_adae_b200 import workloads as wl
    import zxh_adae_b200 as zx

    if not ref_available("cuda"):
        return {"unavailable": "reference CUDA backend not built (oracle/_ref/libzxhref_cuda.so)"}
    out = {"backend": "reference cuda (kernel_cuda.cu, measure_cuda.cu), sm_100a, complex128",
           "method": "header-subtracted execute() wall time, H F F H", "qubits": n, "items": []}
    header = wl.h_all(n)
    hs = Reference(n, backend="cuda")
    hs.push(header)
    hs.execute()

    def ex(sim):
        t0 = time.perf_counter()
        sim.execute()
        return time.perf_counter() - t0

    def item(name, gates, ours_c128, ours_c64, compare=False):
        fs = Reference(n, backend="cuda")
        fs.push(np.concatenate([header, gates]))
        fs.execute()  # first run: allocation and first launches
        h1, f1, f2, h2 = ex(hs), ex(fs), ex(fs), ex(hs)
        t = max(1e-9, 0.5 * ((f1 - h1) + (f2 - h2)))
        rec = {"item": name, "gates": int(len(gates)), "reference_ms": 1e3 * t,
               "reference_GBps": 2 * (1 << n) * 16 / t / 1e9}
        for tag, d in (("c128", ours_c128), ("c64", ours_c64)):
            if d:
                rec[f"ours_{tag}_ms"] = d["ms"]
                rec[f"ours_{tag}_api_ms"] = d["api_ms"]
                rec[f"speedup_{tag}_device"] = 1e3 * t / d["ms"]
                rec[f"speedup_{tag}_api"] = 1e3 * t / d["api_ms"]
        if compare:  # parity at full size: the same gate list through this library
            s = zx.ZXH(n, dtype="complex128", device=local)
            s.push_gates(np.concatenate([header, gates]))
            s.execute()
            ptr, m, eb, g = s.state_view()
            found = fs.device_state()
            if found is None:
                rec["parity"] = "reference state probe failed its layout checks"
            else:
                rptr, rm, rg = found
                rec["parity_live_bits_equal"] = bool(rm == m)
                if rm == m:
                    rec["parity_vs_ours_c128"] = compare_states(_device_state(ptr, m, eb), g,
                                                                _device_state(rptr, rm, 16), rg)
            s.close()
        return fs, rec

    rows = {r["batch"]: r for r in ours.get("config2", {}).get("rows", [])}
    for B in CONFIG2_BATCHES:
        r = rows.get(B, {})
        fs, rec = item(f"diag B={B}", wl.diag_batch(n, B, seed=seed + B), r.get("c128"), r.get("c64"),
                       compare=(B == 4096))
        out["items"].append(rec)
        del fs
    r = rows.get("cascade", {})
    fs, rec = item("cp cascade", wl.cp_cascade(n), r.get("c128"), r.get("c64"))
    out["items"].append(rec)
    del fs
    # a window after a CX chain: the reference runs every CP whose selector spans its
    # lane and high bits as a full sweep of its own (kernel_cuda.cu:767-795,
    # zxh.cpp:535-539); B = 256 keeps that run short
    r = rows.get("cx_chain+256", {})
    fs, rec = item("cx chain, then diag B=256", np.concatenate([wl.cx_chain(n), wl.diag_batch(n, 256, seed=seed + 1)]),
                   r.get("c128"), r.get("c64"), compare=True)
    out["items"].append(rec)
    del fs
    u64, u128 = ours.get("u3_layer"), ours.get("u3_layer_c128")
    conv = (lambda d: {"ms": d["ms_per_layer"], "api_ms": d["api_ms_per_layer"]} if d else None)
    fs, rec = item("U3 layer", wl.u3_layer(n, seed=seed), conv(u128), conv(u64), compare=True)
    out["items"].append(rec)
    # 10^6 shots from the U3-layer state: the reference's measure() (draw + result
    # copy to the host) on the host clock, against this library's measure call
    shots = 1_000_000
    fs.measure(1, shots)
    walls = []
    for k in range(3):
        t0 = time.perf_counter()
        fs.measure(100 + k, shots)
        fs.device_sync()
        walls.append(time.perf_counter() - t0)
    rec = {"item": f"{shots} shots", "reference_ms": 1e3 * min(walls)}
    for tag, key in (("c128", "sampler_c128"), ("c64", "sampler")):
        d = ours.get(key)
        if d:
            rec[f"ours_{tag}_ms"] = d["ms"]
            rec[f"ours_{tag}_api_ms"] = d["api_ms"]
            rec[f"speedup_{tag}_device"] = rec["reference_ms"] / d["ms"]
            rec[f"speedup_{tag}_api"] = rec["reference_ms"] / d["api_ms"]
    out["items"].append(rec)
    del fs, hs
    return out


def run_ours(args):
    world, rank, local, pg = dist_setup(args)
    import zxh_adae_b200 as zx
    from zxh_adae_b200 import workloads as wl

    n, B = args.qubits, args.batch
    dtype = args.dtype
    eb = 8 if dtype == "complex64" else 16
    state = (1 << n) * eb
    peak, peak_kind = peaks()
    if args.workload == "config3":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "workload": "config3", **config3_leg(local)}))
        return
    if args.workload == "config2":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "workload": "config2", **config2_leg(local, n)}))
        return
    if args.workload == "sample":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "workload": "sample",
                              **sampler_leg(local, n, steps=args.steps)}))
        return
    if args.workload == "batch":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "workload": "batch",
                              **batch_leg(local, count=args.batch_count, tune=not args.no_tune)}))
        return
    if args.workload == "adjoint":
        if rank == 0:
            d = adjoint_leg(local, n=n, reps=8, checkpoint_every=48, steps=args.steps, warmup=args.warmup,
                            checks=not args.no_adjoint_checks)
            print(json.dumps({"metric": METRIC, "workload": "adjoint", **d}))
        return
    knobs = [(kv.split("=")[0], int(kv.split("=")[1])) for kv in args.set_param]
    sim = zx.ZXH(n, dtype=dtype, device=local)
    for k, v in knobs:
        sim.set_param(k, v)
    sim.push_gates(wl.h_all(n))
    sim.execute()
    tag = "c64" if dtype == "complex64" else "c128"
    prefix = None
    if args.workload == "u3":
        batches = [wl.u3_layer(n, seed=rank * 100000 + k) for k in range(args.warmup + args.steps)]
        desc = f"U3 layer on all {n} qubits, {dtype}, H-prepared, random angles per step"
        span = dtype == "complex64" and dict(knobs).get("span", 1) != 0
        dominant = "span_kernel" if span else "row_pass_kernel"
        traffic_file = f"span_pass_{n}q_{tag}.md" if span else f"row_pass_{n}q_{tag}.md"
    elif args.workload == "cxwindow":
        # a CX chain first (map updates only): every selector of the windows is then
        # a parity of several real bits, and each window is one Walsh-sum pass
        prefix = wl.cx_chain(n)
        sim.apply(prefix)
        batches = [wl.diag_batch(n, B, seed=rank * 100000 + k) for k in range(args.warmup + args.steps)]
        desc = f"{n}q {dtype}, H-prepared, CX chain, then B={B} random p/cp (50/50) per step"
        dominant, traffic_file = "walsh_kernel", f"walsh_pass_{n}q_{tag}.md"
    else:
        batches = [wl.diag_batch(n, B, seed=rank * 100000 + k) for k in range(args.warmup + args.steps)]
        desc = f"diag-batch {n}q {dtype}, H-prepared, B={B} random p/cp (50/50) per step"
        dominant, traffic_file = "diag_kernel", f"diag_pass_{n}q_{tag}.md"
    dev_ms, launches, passes, wall, clocks = timed_applies(sim, batches, args.warmup, args.steps, pg, local)
    fid = None
    if rank == 0 and world == 1 and not args.no_extras:
        # the same gates in complex128, executed as one list: fidelity error of the timed complex64 state
        ref = zx.ZXH(n, dtype="complex128", device=local)
        ref.push_gates(np.concatenate([wl.h_all(n)] + ([prefix] if prefix is not None else []) + batches))
        ref.execute()
        fid = fidelity_err(sim, ref)
        ref.close()
    sim.close()
    wall_async = timed_async(n, dtype, local, batches, args.warmup, args.steps, pg, prefix, knobs)
    bytes_step = (passes / args.steps) * 2 * state
    dev_total_ms = max_over_ranks(pg, sum(dev_ms), local)
    wall = max_over_ranks(pg, wall, local)
    wall_async = max_over_ranks(pg, wall_async, local)
    value = world * args.steps * bytes_step / (dev_total_ms / 1e3) / 1e9
    e2e_sync = world * args.steps * bytes_step / wall / 1e9
    e2e_value = world * args.steps * bytes_step / wall_async / 1e9
    achieved = bytes_step / (statistics.mean(dev_ms) / 1e3) / 1e9
    traffic = profile_traffic(traffic_file)

    cpu = None
    extras = {}
    if rank == 0 and world == 1:
        if not args.no_cpu_baseline and args.workload == "diag":
            cpu = ref_cpu_sample(3, 1, B)
            if cpu is not None:
                cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        if not args.no_extras and args.workload == "diag":
            extras["config2"] = config2_leg(local, n)
            extras["u3_layer"] = u3_leg(local, n)
            extras["u3_layer_c128"] = u3_leg(local, n, dtype="complex128")
            extras["sampler"] = sampler_leg(local, n)
            extras["sampler_c128"] = sampler_leg(local, n, dtype="complex128")
            extras["config1"] = config1_leg(local)
            extras["config3"] = config3_leg(local)
            extras["adjoint"] = adjoint_leg(local)
            extras["batch"] = batch_leg(local)
            if not args.no_gpu_baseline:
                extras["gpu_baseline"] = gpu_baseline_leg(local, extras, n)
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": tag,
        "data": "synthetic",
        "config": {
            "workload": desc,
            "qubits": n,
            "batch": n if args.workload == "u3" else B,
            "passes_per_step": passes / args.steps,
            "gates_per_s": len(batches[0]) / (dev_total_ms / args.steps / 1e3),
            "passes_per_s": (passes / args.steps) / (dev_total_ms / args.steps / 1e3),
            "state_bytes": state,
            "l2": "state larger than L2, no flush" if state > 126 * 2**20 else "state fits in L2",
            "fidelity_err_vs_complex128": fid,
            "planner_knobs": dict(knobs),
            "parallelism": f"replicas x{world}",
        },
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(len(batches[0]) * 40),
                "d2h_bytes_per_step": 16, "api": "zxh_apply_async + zxh_sync",
                "sync_api_value": e2e_sync},
        "roofline": {
            "kernel": dominant,
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "peak_kind": peak_kind,
            "traffic": traffic,
        },
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "clocks": clocks,
        **extras,
    }
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
