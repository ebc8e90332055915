"""Seeded synthetic particle packings for the operator and solver workloads.

Stands in for hpsint's initial conditions (sintering/initial_values_spherical.h,
initial_values_cloud.h, initial_values_ch_ac.h): spheres (circles in 2D) are
placed so that neighbours overlap by a fixed number of cells, grains that are
close get different order parameters by greedy graph colouring (hpsint colours
with SparsityTools::color_sparsity_pattern, initial_values_cloud.h:208), each
grain is a tanh profile, c is the maximum of the order parameters
(initial_values_ch_ac.h) and mu = 0.

Profile of grain k at distance d from its centre:
    eta_k = 0.5 * (1 - tanh(2 (d - R_k) / width))
so eta goes from 0.88 to 0.12 over one `width` across the surface.
"""
import numpy as np


def place_spheres(dim, box_lo, box_hi, n, radius_sampler, overlap, rng, first_center=None, max_tries=200000):
    """Random sequential packing: every new sphere touches a random earlier one
    with the given overlap (centre distance R_i + R_j - overlap) and overlaps no
    other sphere by more than that."""
    box_lo, box_hi = np.asarray(box_lo, float), np.asarray(box_hi, float)
    centers, radii = [], []
    r0 = radius_sampler(rng)
    c0 = (box_lo + box_hi) / 2 if first_center is None else np.asarray(first_center, float)
    centers.append(c0)
    radii.append(r0)
    tries = 0
    while len(centers) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could only place {len(centers)} of {n} spheres")
        r = radius_sampler(rng)
        j = rng.integers(len(centers))
        v = rng.standard_normal(dim)
        v /= np.linalg.norm(v)
        c = centers[j] + v * (radii[j] + r - overlap)
        if np.any(c - r < box_lo + 1.0) or np.any(c + r > box_hi - 1.0):
            continue
        ok = True
        for ck, rk in zip(centers, radii):
            if np.linalg.norm(c - ck) < rk + r - overlap - 1e-9:
                ok = False
                break
        if ok:
            centers.append(c)
            radii.append(r)
    return np.array(centers), np.array(radii)


def greedy_colouring(centers, radii, buffer):
    """Smallest colour not used by any grain whose surface is closer than `buffer`."""
    n = len(radii)
    colours = -np.ones(n, dtype=int)
    for i in range(n):
        used = set()
        for j in range(n):
            if colours[j] >= 0 and np.linalg.norm(centers[i] - centers[j]) < radii[i] + radii[j] + buffer:
                used.add(colours[j])
        k = 0
        while k in used:
            k += 1
        colours[i] = k
    return colours


def initial_state(dim, n_cells, h, origin, centers, radii, colours, width=2.0, noise=0.0, seed=1):
    """(C, N) nodal state, lexicographic node order (x fastest)."""
    G = int(colours.max()) + 1
    shape = [n_cells[d] + 1 for d in range(dim)]  # x, y(, z)
    N = int(np.prod(shape))
    eta = np.zeros((G,) + tuple(reversed(shape)))  # (G, [nz,] ny, nx)
    coords = [origin[d] + h[d] * np.arange(shape[d]) for d in range(dim)]
    for ck, rk, col in zip(centers, radii, colours):
        # bounding box of the profile (tanh tail below 1e-16 beyond 10 widths)
        lo = [max(0, int(np.floor((ck[d] - rk - 10 * width - origin[d]) / h[d]))) for d in range(dim)]
        hi = [min(shape[d], int(np.ceil((ck[d] + rk + 10 * width - origin[d]) / h[d])) + 1) for d in range(dim)]
        sub = [coords[d][lo[d]:hi[d]] for d in range(dim)]
        grids = np.meshgrid(*reversed(sub), indexing="ij")  # (z,) y, x
        d2 = np.zeros(grids[0].shape)
        for d in range(dim):
            d2 += (grids[dim - 1 - d] - ck[d]) ** 2
        prof = 0.5 * (1.0 - np.tanh(2.0 * (np.sqrt(d2) - rk) / width))
        sl = tuple(slice(lo[d], hi[d]) for d in reversed(range(dim)))
        eta[(col,) + sl] = np.maximum(eta[(col,) + sl], prof)
    u = np.zeros((G + 2, N))
    u[2:] = eta.reshape(G, N)
    u[0] = np.clip(u[2:].max(axis=0), 0.0, 1.0)
    if noise > 0:
        rng = np.random.default_rng(seed)
        u += rng.uniform(-noise, noise, u.shape)
    return u


def operator_bench_packing(n=128, seed=0, n_spheres=8, rmin=12.0, rmax=18.0, overlap=2.0, buffer=16.0):
    """3D operator workload: n^3 unit cells, spheres with radii U[rmin, rmax]
    overlapping by `overlap` cells, grains closer than `buffer` cells coloured
    apart (seed 0 gives 4 order parameters); returns (centers, radii, colours)."""
    rng = np.random.default_rng(seed)
    centers, radii = place_spheres(3, [0, 0, 0], [n, n, n], n_spheres, lambda r: r.uniform(rmin, rmax), overlap, rng)
    colours = greedy_colouring(centers, radii, buffer)
    return centers, radii, colours


def two_particle_2d():
    """2D two-particle case: circles R = 10 at (+-10, 0) on [-40, 40] x [-20, 20]."""
    centers = np.array([[-10.0, 0.0], [10.0, 0.0]])
    radii = np.array([10.0, 10.0])
    return centers, radii, np.array([0, 1])


def colour_with_budget(centers, radii, max_grains, buffers=(32.0, 28.0, 24.0, 20.0, 16.0, 12.0, 8.0, 4.0)):
    """Greedy colouring with the largest buffer (cells between surfaces) whose
    colouring needs at most max_grains order parameters."""
    for buffer in buffers:
        colours = greedy_colouring(centers, radii, buffer)
        if colours.max() + 1 <= max_grains:
            return colours
    raise RuntimeError(f"no colouring with <= {max_grains} order parameters")


def lognormal_packing_3d(n=192, n_spheres=51, median=10.0, sigma=0.2, overlap=2.0, max_grains=10, seed=0):
    """3D solve workload: n^3 unit cells, spheres with lognormal radii
    (median, sigma of log r) in a random sequential packing where every new
    sphere touches an earlier one with a 2-cell overlap, coloured to at most
    max_grains order parameters; returns (centers, radii, colours)."""
    rng = np.random.default_rng(seed)
    centers, radii = place_spheres(3, [0, 0, 0], [n, n, n], n_spheres,
                                   lambda r: float(np.exp(r.normal(np.log(median), sigma))), overlap, rng)
    return centers, radii, colour_with_budget(centers, radii, max_grains)
