"""Grain-tracker particle detection on the device.

Mirrors the detection half of hpsint's GrainTracker::Tracker
(include/pf-applications/grain_tracker/tracker.h:1195-1300) for one order
parameter:
  detect_local_particle_groups  distributed_stitching.h:41-100, :441-480
                                (run_flooding: cells whose largest nodal value
                                exceeds threshold_lower, face-connected)
  compute_particles_info        distributed_stitching.h:264-320
  compute_particles_radii       distributed_stitching.h:322-360
  compute_particles_max_values  distributed_stitching.h:217-258
The labelling runs in the library's CUDA kernels (union-find with
deterministic smallest-cell roots); the tracker's matching of particles to
grains and its remapping decisions stay with the caller, on the small
per-particle tables these functions return.
"""
import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


@dataclass
class Particles:
    """Particles of one order parameter: ids (device int32 tensor per cell, -1 =
    none, cells x fastest) and per particle measure, center, radius, max value."""
    ids: torch.Tensor
    n_particles: int
    measures: np.ndarray = None
    centers: np.ndarray = None
    radii: np.ndarray = None
    max_values: np.ndarray = None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _n_cells(op):
    n = 1
    for d in range(op.mesh.dim):
        n *= int(op.mesh.n_cells[d])
    return n


def detect_local_particle_groups(op, eta, threshold_lower=0.01):
    """Label the particles of the order parameter whose nodal values are the
    device tensor `eta` (N values, e.g. one block of a block vector)."""
    if eta.dtype != torch.float64 or not eta.is_cuda or not eta.is_contiguous():
        raise ValueError("eta must be a contiguous float64 CUDA tensor")
    if eta.numel() < op.N:
        raise ValueError(f"eta holds {eta.numel()} values, the mesh has {op.N} nodes")
    ids = torch.empty(_n_cells(op), dtype=torch.int32, device="cuda")
    n = ctypes.c_int()
    L.check(L.lib().sint_grain_segments(op._h, ctypes.c_void_p(eta.data_ptr()), float(threshold_lower),
                                        ctypes.c_void_p(ids.data_ptr()), ctypes.byref(n), _stream()),
            "sint_grain_segments")
    return Particles(ids, n.value)


def compute_particles_properties(op, eta, particles):
    """Fill measures, centers, radii and max values of `particles` (the
    spherical grain representation)."""
    dim, n = op.mesh.dim, particles.n_particles
    props = np.zeros((n, 3 + dim))
    if n:
        L.check(L.lib().sint_grain_segment_properties(
            op._h, ctypes.c_void_p(eta.data_ptr()), ctypes.c_void_p(particles.ids.data_ptr()), n,
            props.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _stream()), "sint_grain_segment_properties")
    particles.measures = props[:, 0].copy()
    particles.centers = props[:, 1:1 + dim].copy()
    particles.radii = props[:, 1 + dim].copy()
    particles.max_values = props[:, 2 + dim].copy()
    return particles


def detect_particles(op, u, order_parameter, threshold_lower=0.01):
    """Particles of order parameter `order_parameter` of the block vector u
    (the tracker's per-order-parameter loop body, tracker.h:1207-1300)."""
    eta = u[2 + order_parameter]
    return compute_particles_properties(op, eta, detect_local_particle_groups(op, eta, threshold_lower))


def periodicity(op, particles, max_pairs=4096):
    """Distinct pairs (p, q), p <= q, of particles that own cells facing each
    other across a periodic boundary of op (tracker.h:1290-1353); sorted."""
    pairs = (ctypes.c_int * (2 * max_pairs))()
    n = ctypes.c_int()
    L.check(L.lib().sint_grain_segment_periodicity(op._h, ctypes.c_void_p(particles.ids.data_ptr()), pairs,
                                                   max_pairs, ctypes.byref(n), _stream()),
            "sint_grain_segment_periodicity")
    return [(pairs[2 * i], pairs[2 * i + 1]) for i in range(n.value)]


def particle_groups(n_particles, pairs):
    """PeriodicityGraph::build_groups (periodicity_graph.h:57-80): particles
    connected through periodicity pairs form one grain of several segments.
    Returns one group id per particle (-1: not periodic), groups numbered by
    their smallest particle, and the number of groups."""
    parent = list(range(n_particles))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    in_graph = [False] * n_particles
    for p, q in pairs:
        in_graph[p] = in_graph[q] = True
        a, b = find(p), find(q)
        if a != b:
            parent[max(a, b)] = min(a, b)
    groups, ids = {}, []
    for i in range(n_particles):
        if not in_graph[i]:
            ids.append(-1)
            continue
        ids.append(groups.setdefault(find(i), len(groups)))
    return ids, len(groups)


def advection_segments(op, u, threshold_lower=0.01):
    """Segments for the advection mechanism from the state u: every particle
    of every order parameter is one segment (the tracker's grain segments,
    tracker.h:1207-1300, with the particle centers as segment centers).
    Returns (cell_segments: device int32 (n_grains, n_cells), -1 = none;
    centers: device float64 (n_segments, 3); owners: list of (order
    parameter, particle) per segment)."""
    G = op.params.n_grains
    n_cells = _n_cells(op)
    seg = torch.full((G, n_cells), -1, dtype=torch.int32, device="cuda")
    centers, owners, base = [], [], 0
    for b in range(G):
        parts = detect_particles(op, u, b, threshold_lower)
        if parts.n_particles:
            seg[b] = torch.where(parts.ids >= 0, parts.ids + base, parts.ids)
            c = np.zeros((parts.n_particles, 3))
            c[:, :op.mesh.dim] = parts.centers
            centers.append(c)
            owners += [(b, p) for p in range(parts.n_particles)]
            base += parts.n_particles
    cen = np.concatenate(centers) if centers else np.zeros((0, 3))
    return seg, torch.from_numpy(cen).cuda(), owners
