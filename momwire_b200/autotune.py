"""Autotuner for the batched frequency sweep, cached on disk.

The batched complex64 factorisation of a sweep (``mw_zgesv_mixed_batched``)
factors 8, 16 or 32 columns per panel step.  Narrow panels are cheap per
step but need more steps (launches, trailing updates with a short k); wide
panels do fewer, longer steps.  The best width depends on the order n, and
on little else, so the tuner times the candidates once per bucket

    key = (n rounded up to a power of two, degree, ground kind)

on the first structure it meets in that bucket (a short sweep of the real
structure, CUDA events around each candidate), and keeps the winner in a
JSON file: ``$MOMWIRE_B200_TUNE_CACHE``, else
``~/.cache/momwire_b200/autotune.json``.  ``MOMWIRE_B200_AUTOTUNE=0``
turns tuning off (16 columns).
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path

CANDIDATES = (8, 16, 32)
DEFAULT_WIDTH = 16
SMEM_BYTES = 200 * 1024  # the batched panel's shared-memory budget

_lock = threading.Lock()
_cache = None


def cache_path():
    p = os.environ.get("MOMWIRE_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "momwire_b200" / "autotune.json"


def enabled():
    return os.environ.get("MOMWIRE_B200_AUTOTUNE", "1") != "0"


def bucket(n):
    b = 32
    while b < n:
        b *= 2
    return b


def key(n, degree, ground):
    return f"batched_panel/n{bucket(n)}/d{degree}/{ground}"


def feasible(n):
    """Candidate widths whose complex64 panel fits the shared memory."""
    return [w for w in CANDIDATES if n * w * 8 <= SMEM_BYTES]


def _load():
    global _cache
    if _cache is None:
        try:
            _cache = json.loads(cache_path().read_text())
        except (OSError, ValueError):
            _cache = {}
    return _cache


def lookup(k):
    with _lock:
        return _load().get(k)


def record(k, entry):
    with _lock:
        c = _load()
        c[k] = entry
        try:
            path = cache_path()
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_suffix(".tmp")
            tmp.write_text(json.dumps(c, indent=1, sort_keys=True))
            tmp.replace(path)
        except OSError:
            pass  # an unwritable cache only costs re-tuning


def choose(n, degree, ground, time_fn):
    """Panel width for this bucket: cached, else the fastest of the feasible
    candidates by ``time_fn(width) -> ms`` (recorded with the timings)."""
    cands = feasible(n)
    if not cands:
        return DEFAULT_WIDTH
    if not enabled():
        return DEFAULT_WIDTH if DEFAULT_WIDTH in cands else cands[0]
    k = key(n, degree, ground)
    hit = lookup(k)
    if hit is not None and hit.get("width") in cands:
        return int(hit["width"])
    times = {w: float(time_fn(w)) for w in cands}
    best = min(times, key=times.get)
    record(k, {"width": best, "ms": {str(w): round(t, 4) for w, t in times.items()}, "n": int(n)})
    return best
