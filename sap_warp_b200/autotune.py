"""Autotuner of the persistent dense contact solve's launch shape and its
compile-time variants.

The solve kernel is persistent: sms x k CTAs take worlds from a device work
counter, and each world is solved by one CTA, so results do not depend on k
(the resident CTAs per SM).  The kernel is also built in variants of the
LDL^T factorization's column-block width b (sapb_contact_solve_ldlt_blocks):
the best width depends on the DOF count (35 DOFs: seven blocks of 5), and
the width changes the factorization's rounding (not the tolerance the
solve reaches); and a runtime-size kernel with 256 threads per world, which
pays where shared memory leaves one CTA per SM.  The tuner times every
(k, b, threads) on the caller's own first solve (CUDA events, best of a few
runs each) and keeps the fastest in a table keyed by (DOFs per world,
contact-slot bucket, precision, line search, GPU name, SM count), which it
can persist as JSON.  The default shape (the
occupancy bound, the first width) is kept unless another beats it by more
than a margin.
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


def _label(shape) -> str:
    return ",".join(str(int(x)) for x in shape) if isinstance(shape, (tuple, list)) else str(int(shape))


def _shape(value):
    return tuple(int(x) for x in value) if isinstance(value, (tuple, list)) else int(value)


class SolveAutotuner:
    """Choice of launch shape per problem key: an int (resident CTAs per SM)
    or a tuple (CTAs per SM, LDL^T block width[, threads per CTA]).

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

    def lookup(self, key: str):
        entry = self.table.get(key)
        if entry is None:
            return None
        return _shape(entry["choice"]) if "choice" in entry else int(entry["ctas_per_sm"])

    def tune(self, key: str, candidates: list, time_ms: Callable, default=None):
        """The cached choice for `key`, else the candidate with the least time,
        recorded with every candidate's time.  The default (given, or for
        plain ints the largest: the occupancy bound, the launch without
        tuning) is kept unless another beats it by more than `margin` (a
        short sample decides)."""
        known = self.lookup(key)
        if known is not None:
            return known
        cands = [_shape(c) for c in candidates]
        cands = [c for c in dict.fromkeys(cands) if (min(c) if isinstance(c, tuple) else c) >= 1]
        if not cands:
            raise ValueError("no candidate launch shape")
        if default is None:
            default = max(cands) if all(isinstance(c, int) for c in cands) else cands[-1]
        default = _shape(default)
        if default not in cands:
            raise ValueError("the default shape is not a candidate")
        times = {c: min(float(time_ms(c)) for _ in range(self.repeats)) for c in cands}
        best = min(cands, key=lambda c: times[c])
        if times[default] <= times[best] * (1.0 + self.margin):
            best = default
        entry = {"choice": list(best) if isinstance(best, tuple) else best,
                 "ctas_per_sm": best[0] if isinstance(best, tuple) else best,
                 "ms": {_label(c): times[c] for c in cands}}
        self.table[key] = entry
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
