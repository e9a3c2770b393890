"""CPU checks of the host logic behind block SSOR: the DSatur colouring of
the rows inside each block of the row-cached kernel (cn::block_colours) is a
proper colouring of the couplings inside the block up to a few folded rows,
uses few colours, and the
list sizing the kernel and the host agree on (cn::block_list_entries) covers
every in-block coupling of the block exactly once."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import workload
from tool_godot_curvenet_b200 import _lib as L

# C++ entry points of the library's host code (namespace cn, not in the C ABI)
COLOURS = "_ZN2cn13block_coloursEPKiS1_iiPh"
ENTRIES = "_ZN2cn18block_list_entriesEPKiS1_PKhxx"


def _fn(name, restype):
    f = getattr(L.lib(), name)
    f.restype = restype
    return f


def _pattern(oracle, name):
    pos, tris, h, _ = workload(name)
    ap, ac, _ = oracle.System(pos, tris, h, ordering=0, precond=0).export()["A"]
    return np.ascontiguousarray(ap, np.int32), np.ascontiguousarray(ac, np.int32)


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small"])
@pytest.mark.parametrize("rb", [32, 256, 1000, 100000])
def test_dsatur_block_colouring_is_proper(name, rb, oracle):
    ap, ac = _pattern(oracle, name)
    n = ap.size - 1
    col = np.zeros(n, np.uint8)
    nc = _fn(COLOURS, C.c_int)(ap.ctypes.data_as(C.c_void_p), ac.ctypes.data_as(C.c_void_p), n, rb,
                               col.ctypes.data_as(C.c_void_p))
    assert 1 <= nc <= 64 and col.max() + 1 == nc
    maxdeg = int(np.diff(ap).max())
    same = {}
    for i in range(n):
        lo = i // rb * rb
        nb = ac[ap[i]:ap[i + 1]]
        nb = nb[(nb != i) & (nb >= lo) & (nb < lo + rb)]
        same[lo] = same.get(lo, 0) + int(np.sum(col[nb] == col[i]))
    # proper, except where a tiny fourth colour (at most 8 rows) was folded
    # into the lower colours: those rows' couplings to same-colour neighbours
    # are the only ones the sweeps drop
    assert all(v <= 2 * 8 * maxdeg for v in same.values())
    assert sum(same.values()) <= 0.01 * ap[-1]
    # a triangulated surface needs 3 colours; DSatur stays well below the degree bound
    assert nc <= min(maxdeg, 6)


@pytest.mark.parametrize("name", ["cyl_tiny", "torus_small"])
def test_list_entries_cover_every_in_block_coupling(name, oracle):
    ap, ac = _pattern(oracle, name)
    n, rb = ap.size - 1, 512
    col = np.zeros(n, np.uint8)
    _fn(COLOURS, C.c_int)(ap.ctypes.data_as(C.c_void_p), ac.ctypes.data_as(C.c_void_p), n, rb,
                          col.ctypes.data_as(C.c_void_p))
    entries = _fn(ENTRIES, C.c_longlong)
    for blk0 in range(0, n, rb):
        rb_n = min(rb, n - blk0)
        got = entries(ap.ctypes.data_as(C.c_void_p), ac.ctypes.data_as(C.c_void_p),
                      col.ctypes.data_as(C.c_void_p), C.c_longlong(blk0), C.c_longlong(rb_n))
        # per colour: rows x (widest lower + widest upper in-block neighbour count)
        cnt, wl, wu = {}, {}, {}
        couplings = 0
        for i in range(blk0, blk0 + rb_n):
            nb = ac[ap[i]:ap[i + 1]]
            nb = nb[(nb != i) & (nb >= blk0) & (nb < blk0 + rb_n)]
            c = int(col[i])
            lower = int(np.sum(col[nb] < c))
            upper = int(np.sum(col[nb] > c))
            couplings += lower + upper
            cnt[c] = cnt.get(c, 0) + 1
            wl[c] = max(wl.get(c, 0), lower)
            wu[c] = max(wu.get(c, 0), upper)
        want = sum(cnt[c] * (wl[c] + wu[c]) for c in cnt)
        assert got == want
        assert got >= couplings  # every coupling has a slot (padding aside)
