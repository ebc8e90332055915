"""The oracle's assembled Cahn-Hilliard block and its multicolour symmetric
Gauss-Seidel sweeps, pinned on the CPU.

  * the centre blocks of the assembled matrix are the preconditioner's 2x2
    node blocks (oracle_ch_blocks, itself checked against the GPU);
  * with the scalar mobility the matrix applied to (dc, dmu) is the (c, mu)
    rows of the Jacobian-vector product with zero grain directions (the
    preconditioner's Cahn-Hilliard operator and the tangent agree there; the
    tensorial tangent reproduces hpsint's inexact dM/dc, so it differs);
  * the sweeps invert M = (D + L) D^-1 (D + U) in colour order: M z = r.
"""
import numpy as np
import pytest

from helpers import oracle_mesh, particle_state, random_state
from oracle import oracle as O


def neighbours(dim, cells):
    nn = [c + 1 for c in cells] + [1] * (3 - dim)
    N = int(np.prod(nn))
    idx = np.arange(N)
    x, y, z = idx % nn[0], (idx // nn[0]) % nn[1], idx // (nn[0] * nn[1])
    colour = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2)
    out = []
    for k in range(27 if dim == 3 else 9):
        dx, dy, dz = k % 3 - 1, (k // 3) % 3 - 1, (k // 9 - 1 if dim == 3 else 0)
        ok = (x + dx >= 0) & (x + dx < nn[0]) & (y + dy >= 0) & (y + dy < nn[1]) & (z + dz >= 0) & (z + dz < nn[2])
        out.append((ok, np.where(ok, (x + dx) + nn[0] * ((y + dy) + nn[1] * (z + dz)), 0)))
    return out, colour, N


def apply_blocks(A, v, nb, colour, keep):
    out = np.zeros_like(v)
    for k, (ok, j) in enumerate(nb):
        sel = ok & keep(colour[j], colour)
        out[0] += np.where(sel, A[k, 0] * v[0, j] + A[k, 1] * v[1, j], 0.0)
        out[1] += np.where(sel, A[k, 2] * v[0, j] + A[k, 3] * v[1, j], 0.0)
    return out


CASES = [(2, (9, 7), 2), (2, (12, 10), 4), (3, (5, 4, 4), 3), (3, (6, 5, 3), 5)]


@pytest.mark.parametrize("dim,cells,G", CASES)
def test_centre_blocks_are_the_node_blocks(dim, cells, G):
    m, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=True)
    T = O.make_time(40.0, 1.0, [-40.0])
    u = particle_state(dim, cells, G, seed=3)
    A = O.ch_matrix(m, p, T, u)
    assert np.array_equal(A[A.shape[0] // 2], O.ch_blocks(m, p, T, u))


@pytest.mark.parametrize("dim,cells,G", CASES)
def test_matrix_is_the_ch_rows_of_the_tangent(dim, cells, G):
    m, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=False)
    T = O.make_time(40.0, 1.0, [-40.0])
    u = random_state(dim, cells, G, seed=4)
    A = O.ch_matrix(m, p, T, u)
    nb, colour, N = neighbours(dim, cells)
    v = np.random.default_rng(5).standard_normal((G + 2, N))
    v[2:] = 0.0
    jv = O.jvp(m, p, T, u, v)[:2]
    Av = apply_blocks(A, v[:2], nb, colour, lambda cj, ci: np.ones_like(ci, dtype=bool))
    assert np.abs(Av - jv).max() <= 1e-12 * np.abs(jv).max()


@pytest.mark.parametrize("dim,cells,G", CASES)
@pytest.mark.parametrize("tensorial", [False, True])
def test_sweeps_invert_the_gauss_seidel_splitting(dim, cells, G, tensorial):
    m, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=tensorial)
    T = O.make_time(1e3, 1.0, [-1e3])
    u = particle_state(dim, cells, G, seed=6)
    A = O.ch_matrix(m, p, T, u)
    nb, colour, N = neighbours(dim, cells)
    r = np.random.default_rng(7).standard_normal((2, N))
    z = O.ch_sgs(m, A, r)
    D = A[A.shape[0] // 2]
    det = D[0] * D[3] - D[1] * D[2]
    assert np.all(np.abs(det) > 1e-14 * (np.abs(D[0] * D[3]) + np.abs(D[1] * D[2])))
    # (D + U) z = D y, then (D + L) y = r
    w = np.vstack([D[0] * z[0] + D[1] * z[1], D[2] * z[0] + D[3] * z[1]])
    w += apply_blocks(A, z, nb, colour, lambda cj, ci: cj > ci)
    y = np.vstack([(D[3] * w[0] - D[1] * w[1]) / det, (-D[2] * w[0] + D[0] * w[1]) / det])
    back = np.vstack([D[0] * y[0] + D[1] * y[1], D[2] * y[0] + D[3] * y[1]])
    back += apply_blocks(A, y, nb, colour, lambda cj, ci: cj < ci)
    assert np.abs(back - r).max() <= 1e-10 * np.abs(r).max()
