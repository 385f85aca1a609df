"""Autotuner of the solver's tile traits: tile shape and local iterations per
tile visit (the `traits` key), chosen per model, grid size and batch size by
short timed trial solves, with the choice cached on disk.

The reference fixes these traits per model (agd/Eikonal/HFM_CUDA/kernel_traits.py:41-62)
and lets the user override them through `traits`; this build also accepts
`traits='auto'`, which picks, among the compiled tile shapes and a range of
iteration counts, the fastest for problems of this kind.  Every candidate
solves the same discrete scheme to the same stopping test; only the order of
the updates (and hence the float32 roundings) changes.

Cache: a JSON file ($AGD_AUTOTUNE_CACHE, else ~/.cache/agd_b200/autotune.json)
mapping "model|grid bucket|batch bucket|device" to the chosen traits and the
trial times; grid sides and batch sizes are rounded up to powers of two.
"""
import json
import os
import threading

# Compiled tile shapes per model (the visit variants of csrc/sched.cuh) and the
# iteration counts tried with each.
TILE_CANDIDATES = {
    "Riemann2": [(8, 8), (16, 16)],
    "Isotropic2": [(8, 8), (16, 16)],
    "Diagonal2": [(8, 8), (16, 16)],
    "Rander2": [(8, 8)],
    "Riemann3": [(4, 4, 4)],
    "Isotropic3": [(4, 4, 4)],
    "Diagonal3": [(4, 4, 4)],
    "Rander3": [(4, 4, 4)],
}
NITER_CANDIDATES = {2: (4, 6, 8, 12, 16), 3: (2, 4, 6, 8)}

_lock = threading.Lock()


def _pow2(x):
    p = 1
    while p < x:
        p *= 2
    return p


def bucket_key(model, shape, batch, device=""):
    """Cache key: model, grid sides and batch rounded up to powers of two, device name."""
    return "|".join([str(model), "x".join(str(_pow2(int(s))) for s in shape), str(_pow2(int(batch))), str(device)])


def candidates(model):
    nd = int(str(model)[-1])
    return [{"shape_i": tuple(si), "niter_i": n} for si in TILE_CANDIDATES[model] for n in NITER_CANDIDATES[nd]]


class Autotuner:
    """Chooses traits by timing `run(traits) -> seconds` on each candidate (the
    best of `repeats` runs each) and caches the choice under its bucket key."""

    def __init__(self, path=None):
        self.path = path or os.environ.get("AGD_AUTOTUNE_CACHE") or os.path.join(
            os.path.expanduser("~"), ".cache", "agd_b200", "autotune.json")
        self.table = self._load()

    def _load(self):
        try:
            with open(self.path) as f:
                t = json.load(f)
            return t if isinstance(t, dict) else {}
        except (OSError, ValueError):
            return {}

    def _save(self):
        with _lock:
            try:
                os.makedirs(os.path.dirname(self.path), exist_ok=True)
                tmp = self.path + f".{os.getpid()}.tmp"
                with open(tmp, "w") as f:
                    json.dump(self.table, f, indent=1, sort_keys=True)
                os.replace(tmp, self.path)
            except OSError:
                pass  # a read-only home: the choice is still used for this process

    def lookup(self, key):
        e = self.table.get(key)
        if not e:
            return None
        return {"shape_i": tuple(e["shape_i"]), "niter_i": int(e["niter_i"])}

    def tune(self, key, run, cands, repeats=2):
        """The candidate with the smallest time; the entry (choice and times) is cached."""
        times = []
        for c in cands:
            t = min(float(run(c)) for _ in range(repeats))
            times.append((t, c))
        t_best, best = min(times, key=lambda x: x[0])
        self.table[key] = {"shape_i": list(best["shape_i"]), "niter_i": int(best["niter_i"]), "seconds": t_best,
                           "trials": [[list(c["shape_i"]), int(c["niter_i"]), t] for t, c in times]}
        self._save()
        return {"shape_i": tuple(best["shape_i"]), "niter_i": int(best["niter_i"])}, times

    def choose(self, key, run, cands, repeats=2):
        """The cached choice of the bucket, else the tuned one."""
        hit = self.lookup(key)
        if hit is not None:
            return hit, None
        return self.tune(key, run, cands, repeats)
