"""Shared helpers of the test-suite: random sintering states, parity metrics."""
import numpy as np

from oracle import oracle as O


def n_nodes(dim, cells):
    n = 1
    for d in range(dim):
        n *= cells[d] + 1
    return n


def oracle_mesh(dim, cells, h=(1.0, 1.0, 1.0)):
    return O.make_mesh(dim, list(cells) + [0] * (3 - len(cells)), h)


def random_state(dim, cells, G, seed, smooth=True):
    """A (C, N) state with c, eta in [0, 1] and mu in [-1, 1].  With smooth=True
    the fields are sums of a few random Fourier modes (realistic interfaces, all
    mobility branches active) plus small noise; otherwise i.i.d. uniform."""
    rng = np.random.default_rng(seed)
    C = G + 2
    shape = [cells[d] + 1 for d in range(dim)]
    N = int(np.prod(shape))
    if not smooth:
        u = rng.uniform(0.0, 1.0, (C, N))
        u[1] = rng.uniform(-1.0, 1.0, N)
        return u
    axes = np.meshgrid(*[np.linspace(0, 1, s) for s in shape], indexing="ij")
    u = np.zeros((C, N))
    for b in range(C):
        f = np.zeros(shape)
        for _ in range(3):
            k = rng.integers(1, 4, dim)
            ph = rng.uniform(0, 2 * np.pi, dim)
            term = np.ones(shape)
            for d in range(dim):
                term = term * np.cos(np.pi * k[d] * axes[d] + ph[d])
            f += rng.uniform(0.3, 1.0) * term
        f = 0.5 + 0.5 * f / 3.0 + rng.uniform(-0.02, 0.02, shape)
        if b == 1:
            f = 2.0 * f - 1.0
        # numpy meshgrid 'ij' has x first; our node order is x fastest
        u[b] = np.transpose(f).ravel()
    return u


def block_rel_err(ours, ref):
    """max over blocks of |ours_b - ref_b|_2 / |ref_b|_2 (absolute if ref_b == 0)."""
    errs = []
    for b in range(ref.shape[0]):
        nr = np.linalg.norm(ref[b])
        ne = np.linalg.norm(ours[b] - ref[b])
        errs.append(ne / nr if nr > 0 else ne)
    return max(errs)
