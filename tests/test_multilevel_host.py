"""Host set-up of the aggregation hierarchy used by the multilevel flexible-CG pressure solve
(DPM_PSOLVER_MULTILEVEL_FCG), through dpm_multilevel_hierarchy: no device needed.

On the channel's assembled pressure operator (stretched wall-normal spacing) and on a seeded
7-point Neumann box, three pairwise passes per level must coarsen by at least 3x per level down to
a directly solved level of at most 300 rows, keeping the coarse operators sparse.  The host
threads build rows and aggregates in a fixed order and reduce norms over fixed chunks, so the whole
hierarchy (dpm_multilevel_digest) is the same bit for bit on 1, 3 or all host threads."""
import ctypes as C

import numpy as np
import pytest

from dopamine_b200 import cases
from dopamine_b200.solver import lib
from oracle import oracle as O


def ell_from_csr(off, col, val):
    n = off.size - 1
    cnt = np.diff(off)
    W = int(cnt.max())
    ec = np.tile(np.arange(n, dtype=np.int32), (W, 1))
    ev = np.zeros((W, n))
    for s in range(W):
        has = cnt > s
        ec[s, has] = col[off[:-1][has] + s]
        ev[s, has] = val[off[:-1][has] + s]
    return W, np.ascontiguousarray(ec.ravel()), np.ascontiguousarray(ev.ravel())


def hierarchy(n, W, ec, ev, nullsp, passes=3):
    sizes = np.zeros(16, dtype=np.int32)
    nnz = np.zeros(16, dtype=np.int64)
    nl = lib().dpm_multilevel_hierarchy(n, W, ec.ctypes.data_as(C.POINTER(C.c_int)),
                                        ev.ctypes.data_as(C.POINTER(C.c_double)), 1 if nullsp else 0, passes,
                                        sizes.ctypes.data_as(C.POINTER(C.c_int)),
                                        nnz.ctypes.data_as(C.POINTER(C.c_longlong)), 16)
    assert nl > 0, nl
    return sizes[:nl], nnz[:nl]


def digest(n, W, ec, ev, nullsp, passes=3):
    d = C.c_ulonglong()
    nl = lib().dpm_multilevel_digest(n, W, ec.ctypes.data_as(C.POINTER(C.c_int)),
                                     ev.ctypes.data_as(C.POINTER(C.c_double)), 1 if nullsp else 0, passes,
                                     C.byref(d))
    assert nl > 0, nl
    return d.value


def check(sizes, nnz):
    assert sizes[-1] <= 300
    for a, b in zip(sizes[:-1], sizes[1:]):
        assert b * 3 <= a, sizes
    assert np.all(nnz / sizes <= 32), nnz / sizes


def test_channel_operator_hierarchy():
    o = O.Oracle(cases.channel_config(nx=32, ny=24, nz=16, n_steps=1))
    off, col, val = o.poisson_csr()
    n = off.size - 1
    W, ec, ev = ell_from_csr(off, col, val)
    sizes, nnz = hierarchy(n, W, ec, ev, True)
    assert sizes[0] == n and len(sizes) >= 3
    check(sizes, nnz)


def neumann_box_operator():
    """A seeded anisotropic 7-point Neumann operator on a 40x30x20 box, in padded ELL."""
    rng = np.random.default_rng(7)
    nx, ny, nz = 40, 30, 20
    n = nx * ny * nz
    idx = np.arange(n).reshape(nz, ny, nx)
    rows = [[] for _ in range(n)]
    diag = np.zeros(n)
    for ax in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        a, b = idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()
        c = rng.uniform(0.5, 2.0, a.size) * (10.0 if ax == 1 else 1.0)  # anisotropic
        for i, j, v in zip(a.tolist(), b.tolist(), c.tolist()):
            rows[i].append((j, -v))
            rows[j].append((i, -v))
        np.add.at(diag, a, c)
        np.add.at(diag, b, c)
    off = np.zeros(n + 1, dtype=np.int64)
    cols, vals = [], []
    for i in range(n):
        r = sorted(rows[i] + [(i, diag[i])])
        cols += [j for j, _ in r]
        vals += [v for _, v in r]
        off[i + 1] = len(cols)
    W, ec, ev = ell_from_csr(off, np.array(cols, dtype=np.int32), np.array(vals))
    return n, W, ec, ev


def test_neumann_box_hierarchy():
    n, W, ec, ev = neumann_box_operator()
    sizes, nnz = hierarchy(n, W, ec, ev, True)
    check(sizes, nnz)
    # the hierarchy is a pure function of the operator
    s2, z2 = hierarchy(n, W, ec, ev, True)
    assert np.array_equal(sizes, s2) and np.array_equal(nnz, z2)


def _oracle_operator(case):
    off, col, val = O.Oracle(case).poisson_csr()
    return (off.size - 1, *ell_from_csr(off, col, val))


@pytest.mark.parametrize("name", ["channel", "neumann box", "jittered tets"])
def test_same_hierarchy_on_any_thread_count(name):
    from tests.test_host_setup import _Threads
    op = {"channel": lambda: _oracle_operator(cases.channel_config(nx=32, ny=24, nz=16, n_steps=1)),
          "neumann box": neumann_box_operator,
          "jittered tets": lambda: _oracle_operator(cases.hybrid_config(n=10, kind="tet"))}[name]()
    threads = _Threads()
    out = []
    try:
        for t in (1, 3, threads.default):
            threads(t)
            out.append(digest(*op, True))
    finally:
        threads(threads.default)
    assert out[0] == out[1] == out[2], [hex(d) for d in out]
    n, W, ec, ev = op
    ev = ev.copy()
    ev[n + 5] *= 1.01  # the second stored entry of row 5
    assert digest(n, W, ec, ev, True) != out[0]
