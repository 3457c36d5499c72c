"""Autotuner for the back-projector's tile variants.

The back-projector has two single-slice tile variants (``atb_backproject``
flags bits 2-3, ``atb_backproject_batch`` ``variant``): 64 x 64 pixels on
256 threads (variant 0) and 32 x 32 on 128 threads (variant 1, more CTAs per
SM).  Which is faster depends on the image size, the angle count and, for
batches, on how uneven the items are.  The tuner times every candidate on
the device (CUDA events, one warm-up and ``reps`` timed runs) the first time
a workload bucket is seen, and keeps the winner in a JSON cache keyed by
(GPU name, workload kind, size buckets).  Buckets round sizes up to powers
of two, so a cached choice covers every nearby shape.

Cache file: ``$ALGOTOM_B200_AUTOTUNE_CACHE`` or
``~/.cache/algotom_b200/autotune.json``.  A missing or unreadable cache is
treated as empty (and rewritten); writes go through a temporary file and an
atomic rename, under a process-wide lock.  ``ALGOTOM_B200_AUTOTUNE=0``
turns tuning off (variant 0 everywhere).
"""
import json
import os
import threading
import warnings

VARIANTS = (0, 1)

_lock = threading.Lock()
_default = None


def _bucket(n):
    n = max(1, int(n))
    return 1 << (n - 1).bit_length()


def enabled():
    return os.environ.get("ALGOTOM_B200_AUTOTUNE", "1") != "0"


def cache_path():
    p = os.environ.get("ALGOTOM_B200_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "algotom_b200",
                        "autotune.json")


class Autotuner:
    """Times candidates once per key and remembers the fastest."""

    def __init__(self, path=None):
        self.path = path or cache_path()
        self.table = self._load()

    def _load(self):
        try:
            with open(self.path) as f:
                data = json.load(f)
            if not isinstance(data, dict):
                raise ValueError("not a mapping")
            return {str(k): v for k, v in data.items()
                    if isinstance(v, dict) and "choice" in v}
        except FileNotFoundError:
            return {}
        except (OSError, ValueError) as exc:
            warnings.warn("autotune cache %s unreadable (%s); starting empty"
                          % (self.path, exc))
            return {}

    def _save(self):
        d = os.path.dirname(self.path)
        try:
            if d:
                os.makedirs(d, exist_ok=True)
            tmp = "%s.%d.tmp" % (self.path, os.getpid())
            with open(tmp, "w") as f:
                json.dump(self.table, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except OSError as exc:  # a read-only home must not break a run
            warnings.warn("autotune cache %s not written: %s" % (self.path,
                                                                  exc))

    @staticmethod
    def key(kind, gpu, **sizes):
        parts = [kind, gpu] + ["%s=%d" % (k, _bucket(v))
                               for k, v in sorted(sizes.items())]
        return "|".join(parts)

    def choose(self, key, candidates, run):
        """Return the cached choice for ``key`` or time ``run(c)`` (seconds)
        for every candidate, remember the fastest and return it."""
        with _lock:
            hit = self.table.get(key)
            if hit is not None and hit.get("choice") in candidates:
                return hit["choice"]
        times = {}
        for c in candidates:
            times[c] = float(run(c))
        best = min(times, key=times.get)
        with _lock:
            self.table[key] = {"choice": best,
                               "seconds": {str(c): t for c, t in times.items()}}
            self._save()
        return best


def default_tuner():
    global _default
    with _lock:
        if _default is None or _default.path != cache_path():
            _default = Autotuner()
        return _default


def time_device(fn, reps=2):
    """Seconds per call of ``fn`` on the current CUDA stream (1 warm-up)."""
    import torch
    fn()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def _gpu_name():
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def tuned_batch_variant(batch):
    """Tile variant for a :class:`~algotom_b200.rec.batch.BatchedFBP`."""
    if not enabled():
        return 0
    import numpy as np
    rows = np.array([r for r, _ in batch.shapes])
    cols = np.array([c for _, c in batch.shapes])
    key = Autotuner.key("batch", _gpu_name(), items=len(rows),
                        ncol=int(np.median(cols)), nrow=int(np.median(rows)))

    def run(v):
        batch.set_variant(v)
        return time_device(batch.launch)
    return default_tuner().choose(key, VARIANTS, run)


def tuned_single_variant(ncol, nrow, run):
    """Tile variant for one single-slice back-projection; ``run(v)`` must
    perform it with variant ``v``."""
    if not enabled():
        return 0
    key = Autotuner.key("single", _gpu_name(), ncol=ncol, nrow=nrow)
    return default_tuner().choose(key, VARIANTS,
                                  lambda v: time_device(lambda: run(v)))
