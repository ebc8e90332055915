"""Grain-tracker particle detection on the GPU against the CPU oracle.

Particle ids must equal the oracle's flood fill bit for bit (both number
particles in the order a lexicographic cell loop reaches them); measures,
centers and radii agree to 1e-12 relative, maxima exactly.  The hpsint
golden (grain_tracker_elliptical: two grains, spherical representation) is
checked through the CUDA path as well.
"""
import numpy as np
import pytest

from helpers import oracle_mesh, particle_state, tracker_golden_field
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _op(dim, cells, h=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), G=1):
    import hpsint_b200 as hb
    mesh = hb.Mesh(dim, tuple(cells) + (1,) * (3 - len(cells)), tuple(h), tuple(origin))
    return hb.SinteringOperatorGeneric(mesh, hb.Params(G))


def _detect(op, eta_np, thr):
    from hpsint_b200 import grain_tracker as GT
    eta = torch.zeros(op.ld, dtype=torch.float64, device="cuda")
    eta[:op.N] = torch.from_numpy(np.ascontiguousarray(eta_np))
    parts = GT.detect_local_particle_groups(op, eta, thr)
    GT.compute_particles_properties(op, eta, parts)
    return parts


def _compare(dim, cells, eta, thr, h=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    op = _op(dim, cells, h, origin)
    parts = _detect(op, eta, thr)
    om = O.make_mesh(dim, list(cells) + [0] * (3 - len(cells)), h)
    ids_ref, n_ref = O.grain_segments(om, eta, thr)
    assert parts.n_particles == n_ref
    assert np.array_equal(parts.ids.cpu().numpy(), ids_ref)
    props = O.segment_properties(om, eta, ids_ref, n_ref, origin)
    if n_ref:
        assert np.allclose(parts.measures, props[:, 0], rtol=1e-12, atol=0)
        assert np.allclose(parts.centers, props[:, 1:1 + dim], rtol=1e-12, atol=1e-12)
        assert np.allclose(parts.radii, props[:, 1 + dim], rtol=1e-12, atol=0)
        assert np.array_equal(parts.max_values, props[:, 2 + dim])
    return parts, n_ref


def test_golden_elliptical_two_grains(goldens):
    g = goldens["grain_tracker_spherical"]
    dim, cells, h, origin, eta = tracker_golden_field(g)
    parts, n = _compare(dim, cells, eta, g["threshold_lower"], tuple(h) + (1.0,), tuple(origin) + (0.0,))
    assert n == 2
    ours = sorted([list(parts.centers[p]) + [parts.radii[p], parts.max_values[p]] for p in range(n)])
    rtol = 0.5 * 10.0 ** (1 - g["digits"])
    for a, b in zip(ours, sorted(g["segments"])):
        assert np.allclose(a, b, rtol=rtol, atol=0), (a, b)


@pytest.mark.parametrize("dim,cells", [(2, (61, 47)), (3, (29, 23, 17))])
@pytest.mark.parametrize("thr", [0.01, 0.3])
def test_packings_match_oracle(dim, cells, thr):
    G = 6
    u = particle_state(dim, cells, G, seed=31)
    found = 0
    for b in range(G):
        _, n = _compare(dim, cells, u[2 + b], thr, origin=(1.5, -2.0, 0.25))
        found += n
    assert found >= G  # every grain has at least one particle


def test_edge_cases():
    dim, cells = 3, (20, 13, 9)
    N = 21 * 14 * 10
    rng = np.random.default_rng(5)
    # nothing above the threshold
    parts, n = _compare(dim, cells, np.zeros(N), 0.01)
    assert n == 0 and (parts.ids.cpu().numpy() == -1).all()
    # everything one particle
    parts, n = _compare(dim, cells, np.ones(N), 0.01)
    assert n == 1 and (parts.ids.cpu().numpy() == 0).all()
    # sparse noise: many small particles
    _, n = _compare(dim, cells, rng.uniform(0, 1, N) ** 12, 0.9)
    assert n > 20
    # dense noise: a few large, ragged particles (long union chains)
    _, n = _compare(dim, cells, rng.uniform(0, 1, N) ** 6, 0.6)
    assert n >= 1
    # 2D, one cell wide strips touching only at corners: no face contact
    eta = np.zeros((15, 16))
    for k in range(0, 14, 2):
        eta[k, k] = eta[k + 1, k + 1] = 1.0  # a diagonal of cells meeting at corners
    _compare(2, (15, 14), eta.ravel(), 0.5)


def test_labels_are_deterministic():
    dim, cells = 3, (40, 36, 30)
    u = particle_state(dim, cells, 4, seed=37)
    op = _op(dim, cells)
    a = _detect(op, u[2], 0.01)
    b = _detect(op, u[2], 0.01)
    assert a.n_particles == b.n_particles
    assert torch.equal(a.ids, b.ids)
    assert np.array_equal(a.radii, b.radii) and np.array_equal(a.centers, b.centers)


def test_periodic_golden_grains(goldens):
    """grain_tracker_advection_periodic golden (t = 0) through the device
    labelling and pairing: a grain of two segments across the x boundary."""
    from hpsint_b200 import grain_tracker as GT
    from helpers import group_grains, grains_agree, tracker_periodic_golden_fields
    g = goldens["grain_tracker_periodic"]
    dim, cells, h, origin, fields = tracker_periodic_golden_fields(g)
    op = _op(dim, cells, tuple(h) + (1.0,), tuple(origin) + (0.0,))
    op.set_periodicity(g["periodic"])
    grains = []
    for b, eta in enumerate(fields):
        parts = _detect(op, eta, g["threshold_lower"])
        props = np.column_stack([parts.measures, parts.centers, parts.radii, parts.max_values])
        groups, _ = GT.particle_groups(parts.n_particles, GT.periodicity(op, parts))
        grains += group_grains(b, props, groups)
    ref = [(gr["op"], sorted(gr["segments"])) for gr in g["grains"]]
    assert grains_agree(grains, ref, g["digits"]), (grains, ref)


@pytest.mark.parametrize("dim,cells,dirs", [(2, (61, 47), (0, 1)), (3, (29, 23, 17), (0, 2)), (3, (20, 18, 16), (1,))])
def test_periodicity_pairs_match_oracle(dim, cells, dirs):
    from hpsint_b200 import grain_tracker as GT
    # ragged noise particles, many of them cut by the periodic boundaries
    rng = np.random.default_rng(92)
    N = int(np.prod([c + 1 for c in cells]))
    op = _op(dim, cells)
    op.set_periodicity(dirs)
    om = O.make_mesh(dim, list(cells) + [0] * (3 - len(cells)), (1.0, 1.0, 1.0))
    n_pairs = 0
    for b in range(3):
        parts = _detect(op, rng.uniform(0, 1, N) ** 6, 0.6)
        ids = parts.ids.cpu().numpy()
        ref = O.segment_periodicity(om, ids, dirs)
        assert GT.periodicity(op, parts) == ref
        n_pairs += len(ref)
    assert n_pairs > 0  # the packing reaches the periodic boundaries
