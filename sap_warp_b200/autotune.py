"""Autotuner of the persistent dense contact solve's launch shape.

The solve kernel is persistent: sms x k CTAs take worlds from a device work
counter, and each world is solved by one CTA, so results do not depend on k
(the resident CTAs per SM).  The best k is the occupancy maximum for most
shapes, but not for every one (fewer resident worlds share the SM's
instruction cache and issue slots).  The tuner times each k from 1 to the
occupancy bound on the caller's own first solve (CUDA events, best of a few
runs each) and keeps the fastest in a table keyed by (DOFs per world,
contact-slot bucket, precision, line search, GPU name, SM count), which it
can persist as JSON.
"""

from __future__ import annotations

import json
import os
from typing import Callable


def contact_bucket(max_contacts: int) -> int:
    """Contact-slot capacity rounded up to a power of two (at least 8)."""
    b = 8
    while b < int(max_contacts):
        b *= 2
    return b


def tuning_key(dof_per_env: int, max_contacts: int, precision: str, line_search: str, gpu_name: str,
               sm_count: int) -> str:
    gpu = "".join(ch if ch.isalnum() else "_" for ch in str(gpu_name)).strip("_")
    return (f"n{int(dof_per_env)}-c{contact_bucket(max_contacts)}-{precision}-{line_search}-{gpu}-"
            f"{int(sm_count)}sm")


class SolveAutotuner:
    """Choice of resident CTAs per SM per problem key.

    cache_path: a JSON file to load the table from and write it back to after
    each new choice (None: this process only).  repeats: timed runs per
    candidate (the minimum counts)."""

    def __init__(self, cache_path: str | os.PathLike | None = None, repeats: int = 3, margin: float = 0.03):
        self.cache_path = None if cache_path is None else os.fspath(cache_path)
        self.repeats = max(int(repeats), 1)
        self.margin = float(margin)
        self.table: dict = {}
        if self.cache_path and os.path.exists(self.cache_path):
            with open(self.cache_path) as f:
                data = json.load(f)
            if not isinstance(data, dict):
                raise ValueError(f"{self.cache_path}: not an autotuning table")
            self.table = data

    def lookup(self, key: str) -> int | None:
        entry = self.table.get(key)
        return None if entry is None else int(entry["ctas_per_sm"])

    def tune(self, key: str, candidates: list[int], time_ms: Callable[[int], float]) -> int:
        """The cached choice for `key`, else the candidate with the least time,
        recorded with every candidate's time.  The largest candidate (the
        occupancy bound, the launch without tuning) is kept unless another
        beats it by more than `margin` (a short sample decides)."""
        known = self.lookup(key)
        if known is not None:
            return known
        cands = sorted({int(k) for k in candidates if int(k) >= 1})
        if not cands:
            raise ValueError("no candidate launch shape")
        times = {k: min(float(time_ms(k)) for _ in range(self.repeats)) for k in cands}
        best = min(cands, key=lambda k: (times[k], -k))
        if times[cands[-1]] <= times[best] * (1.0 + self.margin):
            best = cands[-1]
        self.table[key] = {"ctas_per_sm": best, "ms": {str(k): times[k] for k in cands}}
        self.save()
        return best

    def save(self) -> None:
        if not self.cache_path:
            return
        d = os.path.dirname(self.cache_path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.table, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)
