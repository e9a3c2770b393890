"""Seeded synthetic meshes, profile-curve cut loops, handles and poses.

The reference measures on character meshes that are not part of its snapshot
(the Mire body meshes); these generators stand in for them with the shapes,
sizes and value distributions of the benchmark configurations:

* cylinder(a, l): ring index i in [0, a), row j in [0, l); vertex id j*a + i;
  theta = 2 pi i / a, z = H j / (l - 1); quad (i, j) splits into
  (v00, v10, v11) and (v00, v11, v01), counter-clockwise seen from outside.
* torus(U, V): major index u in [0, U), minor index v in [0, V); vertex id
  u*V + v; fully periodic; the same quad split.

A cut loop is a closed vertex sequence along mesh edges (a cylinder ring or a
torus meridian).  Handles are picked among vertices that are not on a loop,
so their ids are the same before and after the seam cut; every band between
loops receives at least one handle.  Jitter is i.i.d. N(0, sigma) per
coordinate.  All randomness comes from numpy's PCG64 with the given seed.
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class SynthMesh:
    positions: np.ndarray            # (nv, 3) float64, uncut
    tris: np.ndarray                 # (nt, 3) int32, uncut
    loops: list                      # list of int32 arrays (cut loops)
    band_of: np.ndarray              # (nv,) band id between loops, -1 on a loop
    kind: str = ""
    dims: tuple = ()
    meta: dict = field(default_factory=dict)

    def loop_arrays(self):
        ptr = np.zeros(len(self.loops) + 1, np.int32)
        for i, l in enumerate(self.loops):
            ptr[i + 1] = ptr[i] + len(l)
        verts = np.concatenate(self.loops).astype(np.int32) if self.loops else np.zeros(0, np.int32)
        return ptr, verts


def _quads(rows, cols, wrap_rows, wrap_cols, vid):
    """Triangles of a (rows x cols) quad grid; vid(r, c) gives vertex ids."""
    r_hi = rows if wrap_rows else rows - 1
    c_hi = cols if wrap_cols else cols - 1
    r = np.arange(r_hi)[:, None]
    c = np.arange(c_hi)[None, :]
    v00 = vid(r, c)
    v10 = vid(r, (c + 1) % cols)
    v11 = vid((r + 1) % rows, (c + 1) % cols)
    v01 = vid((r + 1) % rows, c)
    t1 = np.stack([v00, v10, v11], -1).reshape(-1, 3)
    t2 = np.stack([v00, v11, v01], -1).reshape(-1, 3)
    out = np.empty((t1.shape[0] * 2, 3), np.int32)
    out[0::2] = t1
    out[1::2] = t2
    return out


def cylinder(a, l, radius=1.0, height=4.0, sigma=0.01, cut_rows=(), seed=0):
    """Open cylinder a (around) x l (along); cut loops at the given rows."""
    rng = np.random.Generator(np.random.PCG64(seed))
    i = np.arange(a)
    j = np.arange(l)
    th = 2.0 * np.pi * i / a
    pos = np.zeros((l, a, 3))
    pos[:, :, 0] = radius * np.cos(th)[None, :]
    pos[:, :, 1] = radius * np.sin(th)[None, :]
    pos[:, :, 2] = (height * j / (l - 1))[:, None]
    pos = pos.reshape(-1, 3)
    pos += rng.normal(0.0, sigma, pos.shape) if sigma > 0 else 0.0
    tris = _quads(l, a, False, True, lambda r, c: r * a + c)
    loops = [np.arange(a, dtype=np.int32) + r * a for r in cut_rows]
    band = np.searchsorted(np.asarray(sorted(cut_rows)), j, side="right").astype(np.int32)
    band_of = np.repeat(band, a)
    for r in cut_rows:
        band_of[r * a:(r + 1) * a] = -1
    return SynthMesh(pos, tris, loops, band_of, "cylinder", (a, l))


def torus(U, V, R=3.0, r=1.0, sigma=0.005, cut_u=(), seed=0):
    """Torus U (major) x V (minor); cut loops are meridians at major indices cut_u."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = np.arange(U)
    v = np.arange(V)
    th = 2.0 * np.pi * u / U
    ph = 2.0 * np.pi * v / V
    rad = R + r * np.cos(ph)
    pos = np.zeros((U, V, 3))
    pos[:, :, 0] = np.cos(th)[:, None] * rad[None, :]
    pos[:, :, 1] = np.sin(th)[:, None] * rad[None, :]
    pos[:, :, 2] = (r * np.sin(ph))[None, :]
    pos = pos.reshape(-1, 3)
    pos += rng.normal(0.0, sigma, pos.shape) if sigma > 0 else 0.0
    tris = _quads(U, V, True, True, lambda a, b: a * V + b)
    cut_u = sorted(cut_u)
    loops = [np.arange(V, dtype=np.int32) + cu * V for cu in cut_u]
    if cut_u:
        band = (np.searchsorted(np.asarray(cut_u), u, side="right") - 1) % len(cut_u)
    else:
        band = np.zeros(U, np.int64)
    band_of = np.repeat(band.astype(np.int32), V)
    for cu in cut_u:
        band_of[cu * V:(cu + 1) * V] = -1
    return SynthMesh(pos, tris, loops, band_of, "torus", (U, V))


def pick_handles(mesh, fraction, seed):
    """fraction of the vertices (not on a loop), with >= 1 per band; sorted ids."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cand = np.nonzero(mesh.band_of >= 0)[0]
    nv_cut = mesh.positions.shape[0] + sum(len(l) for l in mesh.loops)
    m = max(1, int(round(fraction * nv_cut)))
    m = min(m, cand.size)
    h = set(rng.choice(cand, size=m, replace=False).tolist())
    for b in np.unique(mesh.band_of[cand]):
        members = cand[mesh.band_of[cand] == b]
        if not any(int(x) in h for x in members):
            h.add(int(members[rng.integers(members.size)]))
    return np.array(sorted(h), np.int32)


def rigid_targets(pos, handles, seed, max_angle=np.pi / 4, t_sigma=0.1):
    """Seeded rigid transform of the handle positions about their centroid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    ang = rng.uniform(0.0, max_angle)
    t = rng.normal(0.0, t_sigma, 3)
    Kx = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    Rm = np.eye(3) + np.sin(ang) * Kx + (1 - np.cos(ang)) * Kx @ Kx
    x = pos[handles]
    c = x.mean(axis=0)
    return (x - c) @ Rm.T + c + t


def uniform_targets(pos, handles, half_width, seed, poses=1):
    """rest + U(-w, w) per coordinate; (nh, 3*poses) with pose-major columns."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = pos[handles]
    out = [x + rng.uniform(-half_width, half_width, x.shape) for _ in range(poses)]
    return np.ascontiguousarray(np.concatenate(out, axis=1))


def normal_targets(pos, handles, sigma, seed, poses=1):
    """rest + N(0, sigma) per coordinate; (nh, 3*poses)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = pos[handles]
    out = [x + rng.normal(0.0, sigma, x.shape) for _ in range(poses)]
    return np.ascontiguousarray(np.concatenate(out, axis=1))


# ---------------------------------------------------------------------------
# The five benchmark workloads.

def config1(seed=1):
    """Cylinder 64 x 32, one seam at mid-height (2112 DOF-bearing vertices);
    handles: bottom ring fixed, top ring under a seeded rigid transform."""
    m = cylinder(64, 32, 1.0, 4.0, 0.01, cut_rows=(16,), seed=seed)
    a = 64
    bottom = np.arange(a, dtype=np.int32)
    top = np.arange(a, dtype=np.int32) + 31 * a
    handles = np.concatenate([bottom, top])
    targets = np.concatenate([m.positions[bottom], rigid_targets(m.positions, top, seed + 100)])
    return m, handles, np.ascontiguousarray(targets)


def config2(seed=2):
    """Torus R=3, r=1, 512 (major) x 256 (minor) = 131,072 vertices, 8 seams at
    u = 64 m; 2% handles with U(-0.2, 0.2) displacements."""
    m = torus(512, 256, 3.0, 1.0, 0.005, cut_u=tuple(64 * k for k in range(8)), seed=seed)
    h = pick_handles(m, 0.02, seed + 1)
    return m, h, uniform_targets(m.positions, h, 0.2, seed + 2)


def config5(seed=5):
    """Torus 1024 x 1024 = 1,048,576 vertices, 16 seams; 1% handles, U(-0.5, 0.5)."""
    m = torus(1024, 1024, 3.0, 1.0, 0.0025, cut_u=tuple(64 * k for k in range(16)), seed=seed)
    h = pick_handles(m, 0.01, seed + 1)
    return m, h, uniform_targets(m.positions, h, 0.5, seed + 2)


def config3_mesh(idx, seed=3):
    """Mesh idx of the batch: cylinder or torus by coin flip, n_v log-uniform in
    [2k, 60k] with 2:1 grid aspect, 1-4 seams, 2% handles, 8 poses of N(0, 0.1)."""
    rng = np.random.Generator(np.random.PCG64([seed, idx]))
    is_torus = rng.integers(2) == 1
    nv = float(np.exp(rng.uniform(np.log(2000.0), np.log(60000.0))))
    short = max(8, int(round(np.sqrt(nv / 2.0))))
    long_ = max(8, int(round(nv / short)))
    ns = int(rng.integers(1, 5))
    s = int(rng.integers(1 << 30))
    if is_torus:
        cuts = tuple(sorted({(k * long_) // ns for k in range(ns)}))
        m = torus(long_, short, 3.0, 1.0, 0.005, cut_u=cuts, seed=s)
    else:
        cuts = tuple(sorted({1 + (k + 1) * (long_ - 2) // (ns + 1) for k in range(ns)}))
        m = cylinder(short, long_, 1.0, 4.0, 0.005, cut_rows=cuts, seed=s)
    h = pick_handles(m, 0.02, s + 1)
    return m, h, normal_targets(m.positions, h, 0.1, s + 2, poses=8)


def circle_bezier(center, e1, e2, radius, nseg):
    """Composite cubic Bezier (nseg segments, 3 nseg + 1 points) of the circle
    center + radius (cos phi e1 + sin phi e2); each arc uses the standard
    4/3 tan(dphi/4) tangent length."""
    dphi = 2.0 * np.pi / nseg
    k = 4.0 / 3.0 * np.tan(dphi / 4.0)
    pts = []
    for s in range(nseg):
        p0, p1 = s * dphi, (s + 1) * dphi
        c0 = center + radius * (np.cos(p0) * e1 + np.sin(p0) * e2)
        c1 = center + radius * (np.cos(p1) * e1 + np.sin(p1) * e2)
        t0 = -np.sin(p0) * e1 + np.cos(p0) * e2
        t1 = -np.sin(p1) * e1 + np.cos(p1) * e2
        if s == 0:
            pts.append(c0)
        pts += [c0 + k * radius * t0, c1 - k * radius * t1, c1]
    return np.array(pts)


def config4(seed=4, nseg=5):
    """Torus 128 (major) x 64 (minor) = 8,192 vertices with 4 seams (profile
    curves) at u = 0, 32, 64, 96.  Handles: every loop vertex and its seam copy,
    bound to its loop's curve at tau = nseg * v / 64.  Curves: the meridian
    circles as composite cubic Beziers (nseg = 5 -> 16 control points);
    posed = rest + N(0, 0.05), weights 1 + U(-0.1, 0.1); the target is the
    deformed mesh under parameters perturbed by N(0, 0.02).
    Returns (positions, tris, handles, curve_of, tau, rest_cp, posed_cp,
    weights, target_cp, target_w) on the cut mesh."""
    from .solver import cut_mesh
    U, V, R, r = 128, 64, 3.0, 1.0
    cuts = (0, 32, 64, 96)
    m = torus(U, V, R, r, 0.005, cut_u=cuts, seed=seed)
    tris, parent = cut_mesh(m.positions.shape[0], m.tris, m.loops)
    pos = np.ascontiguousarray(m.positions[parent])
    nv0 = m.positions.shape[0]
    handles, curve_of, tau = [], [], []
    copy = nv0
    for c, cu in enumerate(cuts):
        for v in range(V):
            for vid in (cu * V + v, copy):
                handles.append(vid)
                curve_of.append(c)
                tau.append(nseg * v / V)
            copy += 1
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    rest_cp = []
    for cu in cuts:
        th = 2.0 * np.pi * cu / U
        er = np.array([np.cos(th), np.sin(th), 0.0])
        rest_cp.append(circle_bezier(R * er, er, np.array([0.0, 0.0, 1.0]), r, nseg))
    rest_cp = np.array(rest_cp)
    posed_cp = rest_cp + rng.normal(0.0, 0.05, rest_cp.shape)
    weights = 1.0 + rng.uniform(-0.1, 0.1, len(cuts))
    target_cp = posed_cp + rng.normal(0.0, 0.02, rest_cp.shape)
    target_w = weights + rng.normal(0.0, 0.02, len(cuts))
    return (pos, tris, np.array(handles, np.int32), np.array(curve_of, np.int32), np.array(tau),
            rest_cp, posed_cp, weights, target_cp, target_w)
