"""Autotuner for the tile configuration of each instance size class.

A configuration fixes the tile shape (words per lane / word columns, rows,
planes), the words each thread holds and the subiterations per pass.  The
tuner minimises the engine time of a real batch: starting from the current
table, it visits each size class present in the batch, times the batch with
every configuration of that class's dimensionality (other classes fixed,
median of `reps` runs of the engine stage, CUDA events) and keeps the
fastest; it repeats the sweep `rounds` times.  Winners are written to the
library's table (bgt_tune_set) and cached per GPU name in a JSON file, which
``load_cache`` applies in later processes.

    python -m begputhinning_b200.tune        # tune on the benchmark batch, write the cache
"""
from __future__ import annotations

import ctypes as C
import json
import os
import statistics

from ._lib import check, lib
from .api import Batch, Context, cfg_list

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_cache.json")


def size_class(shape) -> tuple:
    if len(shape) == 2:
        return 2, lib().bgt_tune_class(2, shape[1], shape[0], 1)
    return 3, lib().bgt_tune_class(3, shape[2], shape[1], shape[0])


def current_table() -> dict:
    out = {}
    for dims, n in ((2, 6), (3, 4)):
        for cls in range(n):
            v = C.c_int()
            check(lib().bgt_tune_get(dims, cls, C.byref(v)))
            out[(dims, cls)] = v.value
    return out


def apply(table: dict) -> None:
    for (dims, cls), cfg in table.items():
        check(lib().bgt_tune_set(dims, cls, int(cfg)))


def _time_batch(ctx, tensors_in, tensors_out, cfgs, reps):
    import torch
    torch.cuda.synchronize()
    b = Batch(ctx)
    ids = [b.add(tuple(t.shape), c) for t, c in zip(tensors_in, cfgs)]
    b.finalize()
    for i, ti, to in zip(ids, tensors_in, tensors_out):
        b.set_io(i, ti, to)
    times = []
    for _ in range(reps + 1):
        b.run(graph=True, sync=True)  # the way the batch runs in service
        times.append(b.stage_ms()[1])
    torch.cuda.synchronize()
    b.close()
    return statistics.median(times[1:])


def autotune(items, device: int = 0, reps: int = 5, rounds: int = 1, verbose: bool = False,
             margin: float = 0.01) -> dict:
    """Tune the classes present in `items` (numpy uint8 arrays) on `device`:
    coordinate descent over the size classes, each trial timing the whole
    batch's engine stage (median of `reps` graph runs); a configuration
    replaces the current one only when it is faster by more than `margin`."""
    import torch
    ctx = Context(device)
    tin = [torch.from_numpy(it).to(f"cuda:{device}") for it in items]
    tout = [torch.empty_like(t) for t in tin]
    classes = [size_class(it.shape) for it in items]
    table = current_table()

    def cfg_of(cl):
        v = table.get(cl, -1)
        return v if v >= 0 else -1

    present = sorted(set(classes))
    best_t = _time_batch(ctx, tin, tout, [cfg_of(c) for c in classes], reps)
    for _ in range(rounds):
        for cl in present:
            dims = cl[0]
            best = table.get(cl, -1)
            for cfg in cfg_list(dims):
                trial = dict(table)
                trial[cl] = cfg
                t = _time_batch(ctx, tin, tout, [trial.get(c, -1) for c in classes], reps)
                if verbose:
                    print(f"class {cl} cfg {cfg}: engine {t:.3f} ms", flush=True)
                if t < best_t * (1.0 - margin):  # a change must beat timing noise
                    best_t, best = t, cfg
            table[cl] = best
    ctx.close()
    tuned = {k: v for k, v in table.items() if k in present and v >= 0}
    apply(tuned)
    return {"table": tuned, "engine_ms": best_t}


def gpu_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def save_cache(table: dict, device: int = 0, path: str = CACHE) -> None:
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[gpu_name(device)] = {f"{d}:{c}": int(v) for (d, c), v in table.items()}
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def load_cache(device: int = 0, path: str = CACHE):
    """Apply the cached table of this GPU and return it; None when this GPU
    has no entry.  An empty entry means the tuner kept every default."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        data = json.load(f)
    entry = data.get(gpu_name(device))
    if entry is None:
        return None
    table = {(int(k.split(":")[0]), int(k.split(":")[1])): v for k, v in entry.items()}
    apply(table)
    return table


def main():
    import sys

    from . import synth
    seed = int(sys.argv[1]) if len(sys.argv) > 1 else 3
    imgs, vols = synth.mixed_batch(seed)
    res = autotune(imgs + vols, verbose=True)
    save_cache(res["table"])
    print(json.dumps({"table": {f"{d}:{c}": v for (d, c), v in res["table"].items()},
                      "engine_ms": res["engine_ms"]}))


if __name__ == "__main__":
    main()
