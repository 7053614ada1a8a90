"""What bounds the two-level flexible-CG form's iteration count (design measurement, CPU only).

A numpy restatement of the two-level preconditioner of dopamine_b200/csrc/cuda/fcg.cuh
(z = Z y + S(r - A Z y), y = E^-1 Z^T r, E = Z^T A Z, Z the indicator of P compact parts, S the
part-local Chebyshev of degree 7 on D^-1 A_bb over [0.05, 2]) on the finite-volume Poisson
operator of a 48x32x32 tanh-stretched channel (periodic x and z, walls in y), parts of ~2657 cells
by recursive coordinate bisection as the device kernel uses.  Replacing S by exact solves with
A_bb changes the iteration count by a few percent at most: the coarse space (one value per part),
not the part-local smoother, sets the count.  A stronger local solve cannot bring the two-level
form to twice the plain PCG step on the channel; fewer iterations need a richer coarse space,
which is what the multilevel form provides.
"""
import math

import numpy as np
import pytest

sp = pytest.importorskip("scipy.sparse")
spla = pytest.importorskip("scipy.sparse.linalg")


def _channel_operator(nx, ny, nz, lx=2 * math.pi, ly=2.0, lz=math.pi, stretch=2.0):
    eta = 2.0 * np.arange(ny + 1) / ny - 1.0
    y = 0.5 * ly * np.tanh(stretch * eta) / math.tanh(stretch)
    dx, dz, dy, yc = lx / nx, lz / nz, np.diff(y), 0.5 * (y[1:] + y[:-1])
    n = nx * ny * nz
    I, J, K = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"))

    def idx(i, j, k):
        return i + nx * (j + ny * k)

    c = idx(I, J, K)
    rows, cols, vals = [], [], []
    for nb, cf in ((idx((I + 1) % nx, J, K), dy[J] * dz / dx), (idx(I, J, (K + 1) % nz), dx * dy[J] / dz)):
        rows += [c, nb]; cols += [nb, c]; vals += [-cf, -cf]
    m = J < ny - 1
    cy = dx * dz / (yc[J[m] + 1] - yc[J[m]])
    nb = idx(I[m], J[m] + 1, K[m])
    rows += [c[m], nb]; cols += [nb, c[m]]; vals += [-cy, -cy]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A = (A + sp.diags(-np.asarray(A.sum(axis=1)).ravel())).tocsr()
    cen = np.stack([(I + 0.5) * dx, yc[J], (K + 0.5) * dz], 1)
    return A, cen


def _rcb(cen, P):
    part = np.zeros(len(cen), int)

    def split(ids, p0, np_):
        if np_ == 1:
            part[ids] = p0
            return
        ax = int(np.argmax(cen[ids].max(0) - cen[ids].min(0)))
        o = ids[np.lexsort((ids, cen[ids, ax]))]
        nl = np_ // 2
        cut = int(round(len(ids) * nl / np_))
        split(o[:cut], p0, nl)
        split(o[cut:], p0 + nl, np_ - nl)

    split(np.arange(len(cen)), 0, P)
    return part


def test_coarse_space_bounds_the_two_level_iterations():
    A, cen = _channel_operator(48, 32, 32)
    n = A.shape[0]
    P = round(n / 2657)
    part = _rcb(cen, P)
    Z = sp.csr_matrix((np.ones(n), (np.arange(n), part)), shape=(n, P))
    E = (Z.T @ A @ Z).toarray()
    Einv = np.linalg.inv(E + np.trace(E) / P / P)  # constant mode lifted, as the set-up does
    same = part[A.indices] == np.repeat(part, np.diff(A.indptr))
    Abd = sp.csr_matrix((A.data * same, A.indices.copy(), A.indptr.copy()), shape=(n, n))
    dinv = 1.0 / A.diagonal()
    order = np.argsort(part, kind="stable")
    bounds = np.searchsorted(part[order], np.arange(P + 1))
    blocks = [(order[bounds[b]:bounds[b + 1]],) for b in range(P)]
    lus = [(ids, spla.splu(A[ids][:, ids].tocsc())) for (ids,) in blocks]

    def cheb(rhs, deg=7, lmin=0.05, lmax=2.0):
        th, de = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sig = th / de
        s = dinv * rhs
        d = s / th
        z = np.zeros_like(rhs)
        rho = 1 / sig
        for j in range(deg):
            z += d
            if j == deg - 1:
                break
            s = s - dinv * (Abd @ d)
            rhon = 1 / (2 * sig - rho)
            d = rhon * rho * d + 2 * rhon / de * s
            rho = rhon
        return z

    def exact(rhs):
        out = np.empty_like(rhs)
        for ids, lu in lus:
            out[ids] = lu.solve(rhs[ids])
        return out

    def fcg(b, local, rtol=1e-10, maxit=3000):
        b = b - b.mean()
        r = b.copy()
        bn = np.linalg.norm(b)
        p = q = pq = None
        for it in range(maxit):
            if np.linalg.norm(r) <= rtol * bn:
                return it
            zy = Z @ (Einv @ (Z.T @ r))
            z = zy + local(r - A @ zy)
            z -= z.mean()
            p = z.copy() if p is None else z - (z @ q) / pq * p
            q = A @ p
            pq = p @ q
            al = (z @ r) / pq
            r -= al * q
        return maxit

    b = np.random.default_rng(20261204).standard_normal(n)
    its_cheb, its_exact = fcg(b, cheb), fcg(b, exact)
    print(f"{n} cells, {P} parts: Chebyshev-7 local smoother {its_cheb} iterations, exact part solves {its_exact}")
    assert its_cheb < 3000 and its_exact < 3000
    assert its_exact >= 0.9 * its_cheb
