"""The CPU oracle against hpsint's own golden vectors and known answers.

Mirrors the reference tests
  tests/residual_generic_{scalar,tensorial}_no_rbm.cc  (2x1-cell residual, 4 digits)
  tests/tangent_generic_{scalar,tensorial}.cc          (analytic vs FD tangent)
  tests/free_energy_sintering.cc                        (free-energy KAT, 6 digits)
  tests/power_sum.cc                                    (power sums)
"""
import numpy as np
import pytest

from oracle import oracle as O


def debug_case(g, tensorial):
    m = g["model"]
    mesh = O.make_mesh(2, [2, 1, 0])
    N = O.n_nodes(mesh)
    u = np.zeros((4, N))
    for key, vals in g["debug_state"].items():
        x, y = map(int, key.split(","))
        u[:, x + 3 * y] = vals
    P = O.make_params(2, m["A"], m["B"], m["kappa_c"], m["kappa_p"], m["Mvol"], m["Mvap"],
                      m["Msurf"], m["Mgb"], m["L"], tensorial)
    T = O.make_time(1.0 / m["bdf1_dt"], 1.0, [-1.0 / m["bdf1_dt"]])
    perm = [p[0] + 3 * p[1] for p in g["dealii_dof_points"]]
    return mesh, P, T, u, perm


def agrees_to_digits(ours, gold, digits):
    """True if `ours` rounds to `gold` at `digits` significant digits."""
    ours, gold = np.asarray(ours), np.asarray(gold)
    exp = np.floor(np.log10(np.maximum(np.abs(gold), 1e-300)))
    half_ulp = 0.5 * 10.0 ** (exp - (digits - 1))
    # the printed value was itself rounded: allow one more half unit
    return np.all(np.abs(ours - gold) <= 1.0001 * half_ulp + 1e-300)


@pytest.mark.parametrize("tensorial,key", [(False, "residual_scalar"), (True, "residual_tensorial")])
def test_residual_matches_hpsint_golden(goldens, tensorial, key):
    mesh, P, T, u, perm = debug_case(goldens, tensorial)
    r = O.residual(mesh, P, T, u, [u.copy()], 2)
    ours = r[:, perm]
    gold = np.array(goldens[key])
    assert agrees_to_digits(ours, gold, goldens["residual_digits"]), (ours, gold)


def test_scalar_and_tensorial_goldens_differ_only_in_c_row(goldens):
    s, t = np.array(goldens["residual_scalar"]), np.array(goldens["residual_tensorial"])
    assert not np.allclose(s[0], t[0])
    assert np.allclose(s[1:], t[1:])


@pytest.mark.parametrize("tensorial", [False, True])
def test_tangent_matches_finite_differences(goldens, tensorial):
    """tangent_tester.h:38-106: l1 norm of (analytic - FD) within hpsint's tolerances."""
    mesh, P, T, u, _ = debug_case(goldens, tensorial)
    N = O.n_nodes(mesh)
    n = 4 * N
    eps = goldens["tangent"]["fd_epsilon"]
    r0 = O.residual(mesh, P, T, u, [u.copy()], 2).ravel()
    Ja, Jn = np.zeros((n, n)), np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        Ja[:, j] = O.jvp(mesh, P, T, u, e.reshape(4, N)).ravel()
        up = u.ravel().copy()
        up[j] += eps
        Jn[:, j] = (O.residual(mesh, P, T, up.reshape(4, N), [u.copy()], 2).ravel() - r0) / eps
    l1 = lambda A: np.max(np.sum(np.abs(A), axis=0))  # deal.II FullMatrix::l1_norm
    err = l1(Ja - Jn)
    tol = goldens["tangent"]["tensorial" if tensorial else "scalar"]
    assert err < tol["tol_abs"]
    assert err / l1(Ja) < tol["tol_rel"]
    if not tensorial:
        # the scalar tangent is exact up to FD truncation: much tighter than hpsint's bound
        assert err / l1(Ja) < 1e-8


def test_free_energy_known_answers(goldens):
    kat = goldens["free_energy_kat"]
    G = len(kat["etas"])
    res = O.free_energy(kat["A"], kat["B"], [kat["c"], kat["mu"]] + kat["etas"], G)
    vals = kat["values"]
    checks = [("f", res["f"]), ("df_dc", res["df_dc"]), ("d2f_dc2", res["d2f_dc2"])]
    for i in range(G):
        checks += [(f"df_detai_{i}", res["df_detai"][i]), (f"d2f_dcdetai_{i}", res["d2f_dcdetai"][i]),
                   (f"d2f_detai2_{i}", res["d2f_detai2"][i])]
        for j in range(i + 1, G):
            checks.append((f"d2f_detaidetaj_{i}_{j}", res["d2f_detaidetaj"][i, j]))
    for name, ours in checks:
        gold = vals[name]
        if gold == 0.0:
            assert abs(ours) < 1e-12, name
        else:
            assert agrees_to_digits(ours, gold, kat["digits"]), (name, ours, gold)


def test_power_sum(goldens):
    ps = goldens["power_sum"]
    for section in ("generalized", "optimized"):
        x = ps[section]["input"]
        for p, val in ps[section]["sums"].items():
            assert O.power_sum(x, int(p)) == val


def test_free_energy_derivatives_are_consistent():
    """Second derivatives are the derivatives of the first ones (central FD)."""
    rng = np.random.default_rng(3)
    G = 5
    st = np.concatenate([[0.7, 0.1], rng.uniform(0, 1, G)])
    A, B, h = 16.0, 1.0, 1e-6
    r = O.free_energy(A, B, st, G)
    def fd(k, key, idx=None):
        sp, sm = st.copy(), st.copy()
        sp[k] += h
        sm[k] -= h
        fp, fm = O.free_energy(A, B, sp, G)[key], O.free_energy(A, B, sm, G)[key]
        if idx is not None:
            fp, fm = fp[idx], fm[idx]
        return (fp - fm) / (2 * h)
    assert np.isclose(fd(0, "f"), r["df_dc"], rtol=1e-7)
    assert np.isclose(fd(0, "df_dc"), r["d2f_dc2"], rtol=1e-7)
    for i in range(G):
        assert np.isclose(fd(2 + i, "f"), r["df_detai"][i], rtol=1e-6, atol=1e-8)
        assert np.isclose(fd(0, "df_detai", i), r["d2f_dcdetai"][i], rtol=1e-6, atol=1e-8)
        # d2f_detai2 as coded in hpsint holds the full second derivative
        assert np.isclose(fd(2 + i, "df_detai", i), r["d2f_detai2"][i], rtol=1e-6, atol=1e-8)
        for j in range(G):
            if i != j:
                assert np.isclose(fd(2 + j, "df_detai", i), r["d2f_detaidetaj"][i, j], rtol=1e-6, atol=1e-8)


def test_grain_tracker_segments_match_hpsint_golden(goldens):
    """grain_tracker_elliptical.cc, spherical representation: the flood fill
    (distributed_stitching.h:41-100) finds the two grains, and their centers,
    radii and maxima (:264-395) agree with hpsint's to the printed digits."""
    from helpers import tracker_golden_field
    g = goldens["grain_tracker_spherical"]
    dim, cells, h, origin, eta = tracker_golden_field(g)
    mesh = O.make_mesh(dim, list(cells) + [0], list(h) + [1.0])
    ids, n = O.grain_segments(mesh, eta, g["threshold_lower"])
    assert n == len(g["segments"])
    props = O.segment_properties(mesh, eta, ids, n, list(origin) + [0.0])
    ours = sorted([list(p[1:3]) + [p[3], p[4]] for p in props])
    ref = sorted(g["segments"])
    rtol = 0.5 * 10.0 ** (1 - g["digits"])
    for a, b in zip(ours, ref):
        assert np.allclose(a, b, rtol=rtol, atol=0), (a, b)
    # every cell of a particle is face-connected to it and above the threshold
    assert set(np.unique(ids)) == {-1, 0, 1}


def test_periodic_grain_tracker_matches_hpsint_golden(goldens):
    """grain_tracker_advection_periodic.cc at t = 0: on the periodic mesh the
    particle cut by the x boundary is two particles (no flood across the
    boundary), paired through periodicity (tracker.h:1290-1353) into one grain
    of two segments; all centers, radii and maxima to the printed digits."""
    from hpsint_b200.grain_tracker import particle_groups
    from helpers import group_grains, grains_agree, tracker_periodic_golden_fields
    g = goldens["grain_tracker_periodic"]
    dim, cells, h, origin, fields = tracker_periodic_golden_fields(g)
    mesh = O.make_mesh(dim, list(cells) + [0], list(h) + [1.0])
    grains = []
    for op, eta in enumerate(fields):
        ids, n = O.grain_segments(mesh, eta, g["threshold_lower"])
        props = O.segment_properties(mesh, eta, ids, n, list(origin) + [0.0])
        pairs = O.segment_periodicity(mesh, ids, g["periodic"])
        groups, _ = particle_groups(n, pairs)
        grains += group_grains(op, props, groups)
    ref = [(gr["op"], sorted(gr["segments"])) for gr in g["grains"]]
    assert grains_agree(grains, ref, g["digits"]), (grains, ref)


def rbm_segments(mesh, u, thr):
    """The tracker's particles of each order parameter as advection segments:
    (cell_segments, centers), as the reference's sintering model sets them up
    (sintering_model.h:119, :230)."""
    G = u.shape[0] - 2
    n_cells = int(np.prod([mesh.n[d] for d in range(mesh.dim)]))
    seg = np.full((G, n_cells), -1, dtype=np.int32)
    centers, base = [], 0
    for b in range(G):
        ids, n = O.grain_segments(mesh, u[2 + b], thr)
        props = O.segment_properties(mesh, u[2 + b], ids, n, (0.0, 0.0, 0.0))
        seg[b] = np.where(ids >= 0, ids + base, -1)
        for p in props:
            centers.append(list(p[1:1 + mesh.dim]) + [0.0] * (3 - mesh.dim))
        base += n
    return seg, np.array(centers)


@pytest.mark.parametrize("tensorial,key", [(False, "residual_scalar_rbm"), (True, "residual_tensorial_rbm")])
def test_rbm_residual_matches_hpsint_golden(goldens, tensorial, key):
    """residual_generic_{scalar,tensorial}_rbm: the advection mechanism end to
    end (tracker segments, forces, velocities, advection terms) reproduces
    hpsint's residual to the printed digits."""
    mesh, P, T, u, perm = debug_case(goldens, tensorial)
    a = goldens["rbm"]
    seg, centers = rbm_segments(mesh, u, a["threshold_lower"])
    vft = O.advection_forces(mesh, P, u, seg, centers, (0, 0, 0), a["k"], a["cgb"], a["ceq"], a["smoothening"])
    table = O.advection_velocities(2, vft, centers, a["mt"], a["mr"])
    r = O.residual(mesh, P, T, u, [u.copy()], 2, advection=(seg, table, (0, 0, 0)))
    gold = np.array(goldens[key])
    assert agrees_to_digits(r[:, perm], gold, goldens["residual_digits"]), (r[:, perm], gold)
    # the rigid-body motion changed the eta rows (against the no_rbm golden)
    plain = np.array(goldens[key.replace("_rbm", "")])
    assert not agrees_to_digits(plain, gold, goldens["residual_digits"])
