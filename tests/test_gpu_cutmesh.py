"""Cut-mesh construction on the GPU against the oracle, bit for bit: the
halfedge structure (HalfedgeBuilder.lean:34-90; the oracle restates it and is
pinned by the Halfedge / HalfedgeBuilder / CutAlgorithm examples), the seam
cut (oracle halfedge walk and the product's host fan sweep), and batches of
subdivideEdge / splitFace / insertCrack (CutAlgorithm.lean:49-255) against
the same operations applied one by one by the oracle, with the manifold
invariants checked after each batch."""
import numpy as np
import pytest

from tests.helpers import workload
from tool_godot_curvenet_b200 import CnError, cut_mesh, synth
from tool_godot_curvenet_b200 import cutmesh as G

pytestmark = pytest.mark.gpu

FIXTURE_TRIS = {"triangle": (3, [[0, 1, 2]]), "quad": (4, [[0, 1, 2], [0, 2, 3]]),
                "strip": (4, [[0, 1, 2], [1, 3, 2]])}


def uncut(name):
    if name == "c1":
        m, _, _ = synth.config1()
    elif name == "c2":
        m, _, _ = synth.config2()
    elif name == "c5":
        m, _, _ = synth.config5()
    elif name.startswith("c3_"):
        m, _, _ = synth.config3_mesh(int(name[3:]))
    elif name == "cyl_open":
        m = synth.cylinder(12, 8, cut_rows=(3, 5), seed=21)
    else:
        raise KeyError(name)
    return m


@pytest.mark.parametrize("name", ["triangle", "quad", "strip"])
def test_halfedges_of_spec_fixtures(name, oracle):
    nv, tris = FIXTURE_TRIS[name]
    he = G.halfedges(nv, np.array(tris, np.int32))
    assert np.array_equal(he, oracle.halfedges_from_triangles(nv, np.array(tris, np.int32)))
    assert oracle.manifold(nv, len(tris), he)


@pytest.mark.parametrize("name", ["cyl_open", "c1", "c3_7", "c2", "c5"])
def test_halfedges_bit_exact(name, oracle):
    m = uncut(name)
    nv = m.positions.shape[0]
    he = G.halfedges(nv, m.tris)
    assert np.array_equal(he, oracle.halfedges_from_triangles(nv, m.tris))
    # and on the cut mesh, whose seams add boundaries... of the loops' copies
    tris, parent = cut_mesh(nv, m.tris, m.loops)
    he2 = G.halfedges(parent.size, tris)
    assert np.array_equal(he2, oracle.halfedges_from_triangles(parent.size, tris))


def test_halfedges_first_match_on_duplicate_edges(oracle):
    """A soup with a directed edge used twice (non-manifold): the twin is the
    lowest matching interior index, as the spec's scan finds it."""
    tris = np.array([[0, 1, 2], [0, 1, 3], [1, 0, 4], [2, 1, 5]], np.int32)
    he = G.halfedges(6, tris)
    assert np.array_equal(he, oracle.halfedges_from_triangles(6, tris))


@pytest.mark.parametrize("name", ["cyl_open", "c1", "c3_0", "c3_7", "c2", "c5"])
def test_cut_mesh_gpu_bit_exact(name, oracle):
    m = uncut(name)
    nv = m.positions.shape[0]
    t_gpu, p_gpu = G.cut_mesh_gpu(nv, m.tris, m.loops)
    t_host, p_host = cut_mesh(nv, m.tris, m.loops)
    t_orc, p_orc = oracle.cut_mesh(nv, m.tris, m.loops)
    assert np.array_equal(t_gpu, t_orc) and np.array_equal(p_gpu, p_orc)
    assert np.array_equal(t_gpu, t_host) and np.array_equal(p_gpu, p_host)


def test_cut_mesh_gpu_rejects_an_open_fan(oracle):
    m = uncut("cyl_open")
    nv = m.positions.shape[0]
    # the boundary ring of row 0 with the faces on its left: every sweep from
    # v -> next reaches the halfedge v -> prev, so the oracle's walk accepts
    # it (the copies take all of the ring's faces), and so does the GPU
    ring = np.arange(12, dtype=np.int32)
    t_gpu, p_gpu = G.cut_mesh_gpu(nv, m.tris, [ring])
    t_orc, p_orc = oracle.cut_mesh(nv, m.tris, [ring])
    assert np.array_equal(t_gpu, t_orc) and np.array_equal(p_gpu, p_orc)
    # the same ring reversed: the faces lie on its right, the sweep leaves the
    # mesh through the outer face, and the oracle rejects it too
    with pytest.raises(ValueError):
        oracle.cut_mesh(nv, m.tris, [ring[::-1].copy()])
    with pytest.raises(CnError):
        G.cut_mesh_gpu(nv, m.tris, [ring[::-1].copy()])
    with pytest.raises(CnError):
        G.cut_mesh_gpu(m.positions.shape[0], m.tris, [m.loops[0], m.loops[0]])  # a vertex in two loops


def _apply_sequential(oracle, fn, counts, he, *lists):
    counts = np.asarray(counts, np.int32).copy()
    for args in zip(*lists):
        counts, he = fn(counts, he, *[int(a) for a in args])
        he = he[: counts[2]]
    return counts, he


def _base(oracle, name):
    m = uncut(name)
    nv, nt = m.positions.shape[0], m.tris.shape[0]
    he = oracle.halfedges_from_triangles(nv, m.tris)
    return np.array([nv, nt, he.shape[0]], np.int32), he


@pytest.mark.parametrize("name", ["c1", "c3_7"])
def test_surgery_batches_match_sequential_oracle(name, oracle):
    rng = np.random.default_rng(3)
    counts, he = _base(oracle, name)
    nf = int(counts[1])
    # subdivide one interior halfedge of each of 40 distinct faces (not both
    # directions of an edge), then split each of those faces from the new
    # vertex to the opposite corner
    faces = rng.choice(nf, 40, replace=False)
    edges, taken = [], set()
    for f in faces:
        h = 3 * int(f) + int(rng.integers(3))
        tw = int(he[h, 1])
        if h in taken or tw in taken:
            continue
        taken.update((h, tw))
        edges.append(h)
    c1, h1 = G.subdivide_edges(counts, he, edges)
    c1o, h1o = _apply_sequential(oracle, oracle.subdivide_edge, counts, he, edges)
    assert np.array_equal(c1, c1o) and np.array_equal(h1, h1o)
    assert oracle.manifold(int(c1[0]), int(c1[1]), h1)
    a = [h for h in edges if h1[h, 3] >= 0]
    b = [int(h1[h1[h, 2], 2]) for h in a]  # the halfedge after the new half: target = opposite corner
    c2, h2 = G.split_faces(c1, h1, a, b)
    c2o, h2o = _apply_sequential(oracle, oracle.split_face, c1, h1, a, b)
    assert np.array_equal(c2, c2o) and np.array_equal(h2, h2o)
    assert oracle.manifold(int(c2[0]), int(c2[1]), h2)
    anchors = rng.choice(int(c2[2]), 25, replace=False)
    c3, h3 = G.insert_cracks(c2, h2, anchors)
    c3o, h3o = _apply_sequential(oracle, oracle.insert_crack, c2, h2, anchors)
    assert np.array_equal(c3, c3o) and np.array_equal(h3, h3o)
    for h in anchors:  # each crack lengthens its face loop by 2
        assert oracle.loop_length(h3, int(h)) == oracle.loop_length(h2, int(h)) + 2
