"""Persisted autotuner choices for the batched persistent launch.

``Batch.tune`` (batch.py) times the persistent kernel over its knobs; a
``TuneCache`` keeps the winning settings on disk so later batches of the same
shape on the same GPU model start from them without re-timing. A key is
(dtype, the circuits' qubit-count range, the number of circuits rounded up to a
power of two, GPU name, SM count); the value is the knob settings. The file is
JSON, written atomically (a temporary file renamed over it).

Pure Python: importing this module loads no native code.
"""
from __future__ import annotations

import json
import os
import tempfile
from pathlib import Path

KNOBS = ("grow_regs", "adj_regs", "task_items", "task_elems", "threads")


def batch_key(nqubits, dtype: str, gpu_name: str, sms: int) -> str:
    """Cache key of a batch: dtype, qubit range, circuit count (next power of
    two) and the GPU model."""
    ns = [int(n) for n in nqubits]
    if not ns:
        raise ValueError("a batch has at least one circuit")
    count = 1
    while count < len(ns):
        count <<= 1
    return f"{dtype}|n{min(ns)}-{max(ns)}|c{count}|{gpu_name}|sm{int(sms)}"


class TuneCache:
    """A JSON file of tuned knob settings by batch key."""

    def __init__(self, path) -> None:
        self.path = Path(path)

    def load(self) -> dict:
        try:
            data = json.loads(self.path.read_text())
        except (FileNotFoundError, json.JSONDecodeError):
            return {}
        return data if isinstance(data, dict) else {}

    def get(self, key: str):
        v = self.load().get(key)
        if not isinstance(v, dict) or any(k not in v for k in KNOBS):
            return None
        return {k: int(v[k]) for k in KNOBS}

    def put(self, key: str, settings: dict) -> None:
        data = self.load()
        data[key] = {k: int(settings[k]) for k in KNOBS}
        self.path.parent.mkdir(parents=True, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=str(self.path.parent), prefix=self.path.name, suffix=".tmp")
        try:
            with os.fdopen(fd, "w") as fh:
                json.dump(data, fh, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except BaseException:
            if os.path.exists(tmp):
                os.unlink(tmp)
            raise
