"""CPU-only checks of the product: the C-ABI library loads and exports every
entry point include/curvenet_b200.h declares, the host-only seam cut matches
the oracle's halfedge cut bit for bit, and the GPU entry points fail cleanly
(no crash) without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.conftest import has_gpu
from tool_godot_curvenet_b200 import _lib as L
from tool_godot_curvenet_b200 import cut_mesh, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "curvenet_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cn_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    syms = declared_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(lib, s), s
        assert s in L.SIGNATURES, f"{s} has no ctypes signature"


def test_status_strings():
    assert L.status_string(0) == "ok"
    assert L.status_string(2) == "singular_component"
    assert L.status_string(99) == "unknown"


@pytest.mark.parametrize("cfg", ["c1", "c2", "c3_0", "c3_7", "c5small"])
def test_cut_topology_matches_oracle_bit_exact(cfg, oracle):
    if cfg == "c1":
        m, _, _ = synth.config1()
    elif cfg == "c2":
        m, _, _ = synth.config2()
    elif cfg.startswith("c3"):
        m, _, _ = synth.config3_mesh(int(cfg.split("_")[1]))
    else:
        m = synth.torus(128, 64, cut_u=(0, 16, 32, 48, 64, 80, 96, 112), seed=9)
    nv = m.positions.shape[0]
    t_ours, p_ours = cut_mesh(nv, m.tris, m.loops)
    t_orc, p_orc = oracle.cut_mesh(nv, m.tris, m.loops)
    assert np.array_equal(t_ours, t_orc)
    assert np.array_equal(p_ours, p_orc)
    assert len(p_ours) == nv + sum(len(l) for l in m.loops)
    he = oracle.halfedges_from_triangles(len(p_ours), t_ours)
    assert oracle.manifold(len(p_ours), t_ours.shape[0], he)


def test_cut_rejects_bad_loops():
    m = synth.cylinder(8, 5, cut_rows=(2,), seed=1)
    nv = m.positions.shape[0]
    with pytest.raises(Exception):
        cut_mesh(nv, m.tris, [np.array([16, 18, 20, 22], np.int32)])  # consecutive vertices share no edge
    with pytest.raises(Exception):
        cut_mesh(nv, m.tris, [m.loops[0], m.loops[0]])  # vertex in two loops


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_build_without_device_reports_status():
    m, h, _ = synth.config1()
    t, p = cut_mesh(m.positions.shape[0], m.tris, m.loops)
    pos = np.ascontiguousarray(m.positions[p])
    desc = L.MeshDesc(pos.shape[0], t.shape[0], pos.ctypes.data_as(C.POINTER(C.c_double)),
                      t.ctypes.data_as(C.POINTER(C.c_int32)), h.size, h.ctypes.data_as(C.POINTER(C.c_int32)))
    out = C.c_void_p()
    st = L.lib().cn_build(C.byref(desc), None, C.byref(out))
    assert st in (L.CN_NO_DEVICE, L.CN_CUDA_ERROR)
    assert not out.value


def test_oracle_ic0_breaks_down_after_shift_retries(oracle):
    """The failure-path fixture of tests/test_gpu_failures.py: the oracle's
    IC(0) in colour order meets a non-positive pivot on A and on every shifted
    A + s diag(A), so a build reports CN_NONPOS_PIVOT (3)."""
    from tests.helpers import pivot_breakdown_mesh
    pos, tris, h = pivot_breakdown_mesh()
    assert oracle.System(pos, tris, h, ordering=1).status == 3
    assert oracle.System(pos, tris, h, ordering=1, precond=0).status == 0


def test_surgery_batches_reject_overlapping_records():
    """Batches whose operations would touch one record twice are refused on
    the host, before any device work (no GPU needed)."""
    import ctypes as C
    he = np.array([[1, 5, 1, 0], [2, 4, 2, 0], [0, 3, 0, 0], [2, 2, 4, -1], [1, 1, 5, -1], [0, 0, 3, -1]], np.int32)
    counts = np.array([3, 1, 6], np.int32)
    buf = np.zeros((10, 4), np.int32)
    buf[:6] = he
    IP = C.POINTER(C.c_int32)
    ip = lambda a: a.ctypes.data_as(IP)  # noqa: E731
    edges = np.array([0, 5], np.int32)  # halfedge 0 and its twin 5
    assert L.lib().cn_subdivide_edges(ip(counts), ip(buf), 2, ip(edges)) == L.CN_BAD_INPUT
    anchors = np.array([1, 1], np.int32)
    assert L.lib().cn_insert_cracks(ip(counts), ip(buf), 2, ip(anchors)) == L.CN_BAD_INPUT
    a, b = np.array([0, 1], np.int32), np.array([1, 2], np.int32)  # two splits of face 0
    assert L.lib().cn_split_faces(ip(counts), ip(buf), 2, ip(a), ip(b)) == L.CN_BAD_INPUT
