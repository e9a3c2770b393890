"""The launch-shape autotuner.

Single-mesh systems: cn_autotune times every (lanes per row, threads per
block, blocks) candidate on the device with the caller's right-hand sides
and keeps the fastest; the choice is cached in a JSON file keyed by the
system's size class (rows, nnz per row, levels, preconditioner, precision,
right-hand sides) so later builds of similar systems reuse it.
Batches: BatchSolver candidates (blocks per cluster x threads per block) are
built and timed; the fastest is cached the same way.  Rows per warp of a
batch (lanes per row, 8 or 4 for 24 right-hand sides) are tuned per size
class of mesh inside one handle by tune_batch_lanes.

    python -m tool_godot_curvenet_b200.tune --workload config2 [--sweep]
"""
import argparse
import ctypes as C
import json
import math
import os

import numpy as np

from . import _lib as L
from .solver import BatchSolver, CnError, CutMeshSolver, cut_mesh

# the cache lives in the user's cache directory (CN_TUNE_CACHE overrides),
# not in the package
CACHE = os.environ.get("CN_TUNE_CACHE") or os.path.join(
    os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache"),
    "tool_godot_curvenet_b200", "tuned_shapes.json")


def size_class(info, precond, precision, k):
    return (f"{precond}|{precision}|k{k}|n2^{int(round(math.log2(max(info['n_free'], 1))))}"
            f"|lev{info['n_levels']}|nnz{info['nnz_A'] // max(info['n_free'], 1)}")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(path, d):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def autotune(solver, d_targets, k=3, precond="ic0", reps=3, cache=CACHE, **solve_kw):
    """Tune a CutMeshSolver in place; returns (best, table)."""
    info = solver.info()
    key = size_class(info, precond, solve_kw.get("precision", "mixed"), k)
    o = CutMeshSolver.make_opts(**solve_kw)
    res = (C.c_double * (5 * 120))()
    nres = C.c_int32(0)
    st = L.lib().cn_autotune(solver._h, k, C.c_void_p(d_targets), C.byref(o), reps, res, C.byref(nres))
    if st != L.CN_OK:
        raise CnError(st, "cn_autotune")
    table = [dict(lanes=int(res[5 * i]), block=int(res[5 * i + 1]), grid=int(res[5 * i + 2]),
                  ms=res[5 * i + 3], iterations=int(res[5 * i + 4])) for i in range(nres.value)]
    best = min(table, key=lambda r: r["ms"])
    if cache:
        d = _load(cache)
        d[key] = best
        _save(cache, d)
    return best, table


def apply_cached(solver, precond="ic0", precision="mixed", k=3, cache=CACHE):
    """Set the cached shape of this size class, if any; returns it or None."""
    d = _load(cache)
    best = d.get(size_class(solver.info(), precond, precision, k))
    if best:
        L.lib().cn_set_launch(solver._h, best["lanes"], best["block"], best["grid"])
    return best


def tune_batch(meshes, targets_flat, k=24, shapes=((2, 512), (4, 512), (8, 512), (4, 256), (8, 256)),
               reps=2, **solve_kw):
    """Time BatchSolver shapes (blocks per cluster, threads per block)."""
    import torch
    d_t = torch.from_numpy(targets_flat).cuda()
    out = []
    for cs, blk in shapes:
        with BatchSolver(meshes, k=k, cluster_size=cs, block=blk) as B:
            d_x = torch.empty(int(B.out_off[-1]), dtype=torch.float64, device="cuda")
            B.solve_device(d_t.data_ptr(), d_x.data_ptr(), **solve_kw)
            ms = sorted(B.solve_device(d_t.data_ptr(), d_x.data_ptr(), **solve_kw).device_ms for _ in range(reps))
            out.append(dict(cluster_size=cs, block=blk, clusters=B.info()["n_clusters"], ms=ms[len(ms) // 2]))
    return min(out, key=lambda r: r["ms"]), out


# size classes of the batched meshes (free rows), for the lanes per row
BATCH_CLASSES = (4096, 16384, 1 << 30)


def batch_key(B, precision, classes=BATCH_CLASSES):
    info = B.info()
    n_free = info["n_free"] // max(info["n_meshes"], 1)
    return (f"batch|{precision}|k{info['k']}|m{info['n_meshes']}|avg2^{int(round(math.log2(max(n_free, 1))))}"
            f"|cl{'-'.join(str(c) for c in classes)}")


def tune_batch_lanes(B, d_targets, d_x, precision="mixed", classes=BATCH_CLASSES, reps=3, cache=CACHE,
                     **solve_kw):
    """Rows per warp of a batch, per size class: coordinate descent over the
    classes (each class tried at 4 lanes per row, kept if the whole batch
    launch gets faster, median of `reps` timed launches), starting from 8
    everywhere.  Sets the winner on B and caches it; returns (lanes, table)."""
    key = batch_key(B, precision, classes)
    d = _load(cache) if cache else {}
    if key in d:
        lanes = d[key]["lanes"]
        B.set_lanes(classes, lanes)
        return lanes, d[key]["table"]
    if B.info()["k"] != 24:
        return [1] * len(classes), []

    def timed(lanes):
        B.set_lanes(classes, lanes)
        B.solve_device(d_targets, d_x, precision=precision, **solve_kw)  # capture the graph
        ms = sorted(B.solve_device(d_targets, d_x, precision=precision, **solve_kw).device_ms for _ in range(reps))
        return ms[len(ms) // 2]
    lanes = [8] * len(classes)
    best = timed(lanes)
    table = [dict(lanes=list(lanes), ms=best)]
    for c in range(len(classes)):
        trial = list(lanes)
        trial[c] = 4
        ms = timed(trial)
        table.append(dict(lanes=list(trial), ms=ms))
        if ms < best:
            best, lanes = ms, trial
    B.set_lanes(classes, lanes)
    if cache:
        d[key] = dict(lanes=lanes, ms=best, table=table)
        _save(cache, d)
    return lanes, table


def main():
    import torch

    from . import synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="config2", choices=["config1", "config2", "config5"])
    ap.add_argument("--precond", default="ic0", choices=["ic0", "jacobi", "hsc"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--sweep", action="store_true", help="print every candidate")
    ap.add_argument("--no-cache", action="store_true")
    a = ap.parse_args()
    m, h, t = getattr(synth, a.workload)()
    tris, parent = cut_mesh(m.positions.shape[0], m.tris, m.loops)
    pos = np.ascontiguousarray(m.positions[parent])
    with CutMeshSolver(pos, tris, h, precond=a.precond) as s:
        d_t = torch.from_numpy(np.ascontiguousarray(t[:, :3])).cuda()
        best, table = autotune(s, d_t.data_ptr(), 3, a.precond, cache=None if a.no_cache else CACHE,
                               mode="deform", precision=a.precision, tol=1e-8)
    if a.sweep:
        for r in sorted(table, key=lambda r: r["ms"]):
            print(json.dumps(dict(workload=a.workload, precond=a.precond, precision=a.precision, **r)))
    print(json.dumps(dict(best=best)))


if __name__ == "__main__":
    main()
