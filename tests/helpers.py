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


def random_gradients(nh, seed, scale=0.15):
    """(nh, 9) per-handle deformation gradients R (I + scale N(0, 1))."""
    rng = np.random.default_rng(seed)
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    ang = rng.uniform(0, np.pi / 3)
    Kx = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R = np.eye(3) + np.sin(ang) * Kx + (1 - np.cos(ang)) * Kx @ Kx
    F = np.stack([R @ (np.eye(3) + scale * rng.normal(size=(3, 3))) for _ in range(nh)])
    return F.reshape(nh, 9)


def sample_col(nv, h):
    sc = np.full(nv, -1, np.int32)
    sc[h] = np.arange(h.size, dtype=np.int32)
    return sc


def composed_deformation(oracle, pos, tris, h, Fc, Xc):
    """DeformSolve.lean:110-135 composed from oracle pieces: the oracle's
    k = 9 harmonic solve (CG to 1e-14), the bridge in numpy over the oracle's
    per-face cot Laplacian, Stage 2 by a sparse direct solve of the oracle's
    A.  Handles overlaid with X_c."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    nv = pos.shape[0]
    ref = oracle.System(pos, tris, h)
    st, Fv, _, _ = ref.solve(Fc, mode=0, tol=1e-14)
    assert st == 0
    Fv = Fv.copy()
    Fv[h] = Fc  # harmonic overlay of the handles (computeFh :40-53)
    rest = pos
    cx = np.zeros((nv, 3))
    cx[h] = Xc
    rhs = np.zeros((nv, 3))
    for f, (a, b, c) in enumerate(tris):
        corners = (b, c, a)  # faceLoop order t1, t2, t0
        Ff = (Fv[b] + Fv[c] + Fv[a]) / 3.0
        Fm = Ff.reshape(3, 3)
        Lf = oracle.triangle_cot_laplacian(pos[corners[0]], pos[corners[1]], pos[corners[2]])
        diff = np.stack([cx[v] - Fm @ rest[v] for v in corners])
        contrib = Lf @ diff
        for q, v in enumerate(corners):
            rhs[v] -= contrib[q]
    e = ref.export()
    free_of = e["free_of"]
    Ap, Ac, Av = e["A"]
    A = sp.csr_matrix((Av, Ac, Ap), shape=(free_of.size, free_of.size))
    x = np.zeros((nv, 3))
    x[free_of] = spl.spsolve(A.tocsc(), rhs[free_of])
    x[h] = Xc
    return x


def pivot_breakdown_mesh(seed=2566):
    """A planar 8 x 8 grid with in-plane jitter U(-0.49, 0.49) and x stretched
    by a seeded factor: its obtuse triangles give large positive off-diagonal
    entries, and IC(0) of the reduced matrix in colour order meets a
    non-positive pivot on A and on A + s diag(A) for every retry shift s.
    Handles: the first row.  Returns (positions, tris, handles)."""
    from tool_godot_curvenet_b200 import synth
    rng = np.random.default_rng(seed)
    a, l = int(rng.integers(4, 10)), int(rng.integers(4, 10))
    xs, ys = np.meshgrid(np.arange(a, dtype=float), np.arange(l, dtype=float))
    pos = np.stack([xs.ravel(), ys.ravel(), np.zeros(a * l)], 1)
    pos[:, :2] += rng.uniform(-0.49, 0.49, (a * l, 2))
    pos[:, 0] *= float(rng.uniform(0.05, 20))
    tris = synth._quads(l, a, False, False, lambda r, c: r * a + c)
    return np.ascontiguousarray(pos), tris, np.arange(a, dtype=np.int32)


def line_curve(p0, p1, nseg=1):
    """A composite cubic Bezier of nseg segments along the straight line p0 -> p1
    (control points at thirds), (3 nseg + 1, 3)."""
    p0, p1 = np.asarray(p0, float), np.asarray(p1, float)
    s = np.linspace(0.0, 1.0, 3 * nseg + 1)
    return p0[None, :] + s[:, None] * (p1 - p0)[None, :]


def star_curvenet(nh, n_samples=6, seed=0):
    """Intersection test net: four open curves leaving one node along +x, +y,
    -x, -y (counter-clockwise), each bent by seeded control-point noise, plus
    a triangle of three curves whose corners are three more nodes (both ends
    of each curve at a node), plus a T-junction (two anti-parallel curves and
    one perpendicular).  Handles 0..nh-1 are bound round-robin to (curve,
    sample, side); every 7th stays unbound.  Returns (net dict, rest_cp)."""
    rng = np.random.default_rng(seed)
    curves = []
    for d in ([1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0]):
        curves.append(line_curve([0, 0, 0], np.asarray(d, float) * 2.0, 2))
    tri = [np.array([3.0, 0.0, 0.2]), np.array([4.0, 1.5, 0.0]), np.array([2.5, 1.2, -0.3])]
    for i in range(3):
        curves.append(line_curve(tri[i], tri[(i + 1) % 3], 2))
    c0 = np.array([0.0, -3.0, 0.0])
    curves.append(line_curve(c0, c0 + [1.5, 0, 0], 2))
    curves.append(line_curve(c0, c0 + [0, 1.5, 0], 2))
    curves.append(line_curve(c0, c0 + [-1.5, 0, 0], 2))
    rest_cp = np.array(curves)
    # interior control points bent a little (ends stay on the nodes)
    rest_cp[:, 1:-1] += rng.normal(0.0, 0.05, rest_cp[:, 1:-1].shape)
    C = rest_cp.shape[0]
    S = (rest_cp.shape[1] - 1) // 3
    tau = np.tile(np.linspace(0.0, S, n_samples), (C, 1))
    node_ptr = [0, 4, 6, 8, 10, 13]
    node_ends = [2 * 0, 2 * 1, 2 * 2, 2 * 3,                  # star centre, CCW
                 2 * 4 + 0, 2 * 6 + 1, 2 * 5 + 0, 2 * 4 + 1,  # triangle corners
                 2 * 6 + 0, 2 * 5 + 1,
                 2 * 7, 2 * 8, 2 * 9]                          # T-junction: +x, +y, -x
    hc = np.array([(h % C) if h % 7 else -1 for h in range(nh)], np.int32)
    hs = np.array([(h // C) % n_samples for h in range(nh)], np.int32)
    hd = np.array([(h // (C * n_samples)) % 2 for h in range(nh)], np.int32)
    net = dict(rest_cp=rest_cp, sample_tau=tau, closed=np.zeros(C, np.int32), node_ptr=np.array(node_ptr, np.int32),
               node_ends=np.array(node_ends, np.int32), handle_curve=hc, handle_sample=hs, handle_side=hd)
    return net, rest_cp


def loop_curvenet(seed=4, nseg=5):
    """The adjoint workload's torus 128 x 64 with its 4 seams as closed
    profile curves (isolated): every seam vertex and its copy bound to its
    curve's sample (plus side for the original, minus for the copy).
    Returns (positions, tris, handles, net dict)."""
    from tool_godot_curvenet_b200 import synth
    pos, tris, h, cof, tau, rest_cp, _, _, _, _ = synth.config4(seed, nseg)
    V = 64
    samples = np.tile(nseg * np.arange(V) / V, (rest_cp.shape[0], 1))
    hs = np.rint(np.asarray(tau) * V / nseg).astype(np.int32)
    hd = np.tile(np.array([0, 1], np.int32), h.size // 2)
    net = dict(rest_cp=rest_cp, sample_tau=samples, closed=np.ones(rest_cp.shape[0], np.int32),
               node_ptr=np.zeros(1, np.int32), node_ends=np.zeros(0, np.int32), handle_curve=np.asarray(cof, np.int32),
               handle_sample=hs, handle_side=hd)
    return pos, tris, h, net
