"""Shared workload helpers for the tests."""
import functools

import numpy as np

from tool_godot_curvenet_b200 import cut_mesh, synth


@functools.lru_cache(maxsize=None)
def workload(name):
    """(positions, tris, handles, targets) of a cut mesh."""
    if name == "c1":
        m, h, t = synth.config1()
    elif name == "c2":
        m, h, t = synth.config2()
    elif name == "c5":
        m, h, t = synth.config5()
    elif name.startswith("c3_"):
        m, h, t = synth.config3_mesh(int(name[3:]))
    elif name == "torus_small":
        m = synth.torus(96, 48, cut_u=(0, 24, 48, 72), seed=11)
        h = synth.pick_handles(m, 0.02, 12)
        t = synth.uniform_targets(m.positions, h, 0.2, 13)
    elif name == "torus_mid":
        m = synth.torus(160, 112, cut_u=(0, 40, 80, 120), seed=31)
        h = synth.pick_handles(m, 0.02, 32)
        t = synth.uniform_targets(m.positions, h, 0.2, 33)
    elif name == "cyl_tiny":
        m = synth.cylinder(12, 8, cut_rows=(4,), seed=21)
        h = np.concatenate([np.arange(12), np.arange(12) + 7 * 12]).astype(np.int32)
        t = synth.rigid_targets(m.positions, h, 22)
    else:
        raise KeyError(name)
    tris, parent = cut_mesh(m.positions.shape[0], m.tris, m.loops)
    pos = np.ascontiguousarray(m.positions[parent])
    return pos, tris, np.asarray(h, np.int32), np.ascontiguousarray(t)


def csr_to_dict(ptr, col, val, rows_map=None, cols_map=None):
    """{(row_id, col_id): value} with optional relabelling."""
    out = {}
    n = ptr.size - 1
    for i in range(n):
        r = rows_map[i] if rows_map is not None else i
        for e in range(ptr[i], ptr[i + 1]):
            c = cols_map[col[e]] if cols_map is not None else col[e]
            out[(int(r), int(c))] = val[e]
    return out


def rel_err(x, ref):
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))
