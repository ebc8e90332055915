"""ctypes binding of the CPU oracle (test infrastructure only).

Loaded by the test-suite, the smoke check and the CPU-baseline leg of the
benchmark to check or time the CUDA operator; nothing in the product imports
it.  Vectors are numpy float64 arrays of shape (C, N) in the lexicographic
SoA layout described in sint_oracle.cpp.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsint_oracle.so")

_c_int, _c_double, _c_void = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


class Mesh(ctypes.Structure):
    _fields_ = [("dim", _c_int), ("n", _c_int * 3), ("h", _c_double * 3)]


class Params(ctypes.Structure):
    _fields_ = [("n_grains", _c_int), ("A", _c_double), ("B", _c_double),
                ("kappa_c", _c_double), ("kappa_p", _c_double),
                ("Mvol", _c_double), ("Mvap", _c_double), ("Msurf", _c_double),
                ("Mgb", _c_double), ("L", _c_double), ("tensorial", _c_int)]


class Advection(ctypes.Structure):
    _fields_ = [("cell_segments", ctypes.POINTER(_c_int)), ("segments", ctypes.POINTER(_c_double)),
                ("n_segments", _c_int), ("origin", _c_double * 3)]


class Time(ctypes.Structure):
    _fields_ = [("w0", _c_double), ("w_alg", _c_double), ("order", _c_int),
                ("w_hist", _c_double * 4)]


_lib = None


def build():
    """Compile the oracle library with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        L.oracle_free_energy.argtypes = [_c_double, _c_double, P(_c_double), _c_int, P(_c_double)]
        L.oracle_power_sum.argtypes = [P(_c_double), _c_int, _c_int]
        L.oracle_power_sum.restype = _c_double
        U16 = P(ctypes.c_uint16)
        L.oracle_residual.argtypes = [P(Mesh), P(Params), P(Time), P(_c_double), P(P(_c_double)),
                                      _c_int, U16, P(Advection), P(_c_double), _c_int]
        L.oracle_jvp.argtypes = [P(Mesh), P(Params), P(Time), P(_c_double), P(_c_double),
                                 U16, P(Advection), P(_c_double), _c_int]
        L.oracle_ac_diagonal.argtypes = [P(Mesh), P(Params), P(Time), P(_c_double), U16, P(Advection), P(_c_double),
                                         _c_int]
        L.oracle_ch_blocks.argtypes = [P(Mesh), P(Params), P(Time), P(_c_double), U16, P(Advection), P(_c_double),
                                       _c_int]
        L.oracle_ch_matrix.argtypes = [P(Mesh), P(Params), P(Time), P(_c_double), U16, P(Advection), P(_c_double),
                                       _c_int]
        L.oracle_ch_sgs.argtypes = [P(Mesh), P(_c_double), P(_c_double), P(_c_double)]
        L.oracle_grain_mask.argtypes = [P(Mesh), P(Params), P(_c_double), _c_double, U16]
        L.oracle_grain_segments.argtypes = [P(Mesh), P(_c_double), _c_double, P(_c_int), P(_c_int)]
        L.oracle_segment_properties.argtypes = [P(Mesh), P(_c_double), P(_c_double), P(_c_int), _c_int,
                                                P(_c_double)]
        L.oracle_advection_forces.argtypes = [P(Mesh), P(Params), P(_c_double), P(_c_double), U16, P(_c_int),
                                              P(_c_double), _c_int, _c_double, _c_double, _c_double, _c_double,
                                              P(_c_double)]
        L.oracle_advection_velocities.argtypes = [_c_int, P(_c_double), P(_c_double), _c_int, _c_double,
                                                  _c_double, P(_c_double)]
        L.oracle_advection_courant.argtypes = [P(Mesh), P(Params), U16, P(Advection), _c_double]
        _lib = L
    return _lib


def _dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(_c_double))


def _mptr(mask, mesh):
    """Cell-mask argument: None (every grain) or uint16 per cell."""
    if mask is None:
        return None, None
    n = 1
    for d in range(mesh.dim):
        n *= mesh.n[d]
    m = np.ascontiguousarray(mask, dtype=np.uint16).reshape(-1)
    assert m.size == n, (m.size, n)
    return m, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))


def make_mesh(dim, cells, h=(1.0, 1.0, 1.0)):
    m = Mesh()
    m.dim = dim
    for d in range(3):
        m.n[d] = int(cells[d]) if d < dim else 0
        m.h[d] = float(h[d]) if d < dim else 1.0
    return m


def make_params(n_grains, A=16.0, B=1.0, kappa_c=1.0, kappa_p=0.5, Mvol=1e-2, Mvap=1e-10,
                Msurf=4.0, Mgb=0.4, L=1.0, tensorial=True):
    return Params(n_grains, A, B, kappa_c, kappa_p, Mvol, Mvap, Msurf, Mgb, L, int(bool(tensorial)))


def make_time(w0, w_alg=1.0, w_hist=()):
    t = Time()
    t.w0, t.w_alg, t.order = float(w0), float(w_alg), len(w_hist)
    for i, w in enumerate(w_hist):
        t.w_hist[i] = float(w)
    return t


def n_nodes(mesh):
    n = 1
    for d in range(mesh.dim):
        n *= mesh.n[d] + 1
    return n


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


def free_energy(A, B, state, G):
    st = np.ascontiguousarray(state, dtype=np.float64)
    out = np.zeros(2 + 3 * G + G * G + 1)
    _check(lib().oracle_free_energy(A, B, _dptr(st), G, _dptr(out)), "free_energy")
    k = 0
    res = {"f": out[0], "df_dc": out[1]}
    k = 2
    res["df_detai"] = out[k:k + G].copy(); k += G
    res["d2f_dc2"] = out[k]; k += 1
    res["d2f_dcdetai"] = out[k:k + G].copy(); k += G
    res["d2f_detai2"] = out[k:k + G].copy(); k += G
    res["d2f_detaidetaj"] = out[k:k + G * G].reshape(G, G).copy()
    return res


def power_sum(x, p):
    xs = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oracle_power_sum(_dptr(xs), len(xs), p)


def n_cells(mesh):
    n = 1
    for d in range(mesh.dim):
        n *= mesh.n[d]
    return n


def grain_mask(mesh, params, u, tol):
    """Cell masks of the grain cut-off (uint16 per cell, bit b = grain b relevant)."""
    C, N = params.n_grains + 2, n_nodes(mesh)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(C, N)
    m = np.zeros(n_cells(mesh), dtype=np.uint16)
    _check(lib().oracle_grain_mask(ctypes.byref(mesh), ctypes.byref(params), _dptr(u), float(tol),
                                   m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))), "grain_mask")
    return m


def _adv(adv, mesh):
    """Advection argument: None or (cell_segments (G, n_cells) int, segments (S, 9), origin)."""
    if adv is None:
        return None, None
    seg = np.ascontiguousarray(adv[0], dtype=np.int32)
    data = np.ascontiguousarray(adv[1], dtype=np.float64).reshape(-1, 9)
    a = Advection()
    a.cell_segments = seg.ctypes.data_as(ctypes.POINTER(_c_int))
    a.segments = data.ctypes.data_as(ctypes.POINTER(_c_double))
    a.n_segments = data.shape[0]
    org = list(adv[2]) + [0.0] * (3 - len(adv[2]))
    for d in range(3):
        a.origin[d] = float(org[d])
    return (seg, data), ctypes.byref(a)


def residual(mesh, params, time, u, hist=(), with_td=2, threads=0, mask=None, advection=None):
    C, N = params.n_grains + 2, n_nodes(mesh)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(C, N)
    hs = [np.ascontiguousarray(h, dtype=np.float64).reshape(C, N) for h in hist]
    arr = (ctypes.POINTER(_c_double) * max(1, len(hs)))(*[_dptr(h) for h in hs])
    dst = np.zeros((C, N))
    keep, mp = _mptr(mask, mesh)
    keep_a, ap = _adv(advection, mesh)
    _check(lib().oracle_residual(ctypes.byref(mesh), ctypes.byref(params), ctypes.byref(time), _dptr(u),
                                 arr, with_td, mp, ap, _dptr(dst), threads or os.cpu_count()), "residual")
    return dst


def jvp(mesh, params, time, lin, src, threads=0, mask=None, advection=None):
    C, N = params.n_grains + 2, n_nodes(mesh)
    lin = np.ascontiguousarray(lin, dtype=np.float64).reshape(C, N)
    src = np.ascontiguousarray(src, dtype=np.float64).reshape(C, N)
    dst = np.zeros((C, N))
    keep, mp = _mptr(mask, mesh)
    keep_a, ap = _adv(advection, mesh)
    _check(lib().oracle_jvp(ctypes.byref(mesh), ctypes.byref(params), ctypes.byref(time), _dptr(lin), _dptr(src),
                            mp, ap, _dptr(dst), threads or os.cpu_count()), "jvp")
    return dst


def ac_diagonal(mesh, params, time, lin, threads=0, mask=None, advection=None):
    C, N, G = params.n_grains + 2, n_nodes(mesh), params.n_grains
    lin = np.ascontiguousarray(lin, dtype=np.float64).reshape(C, N)
    d = np.zeros((G, N))
    keep, mp = _mptr(mask, mesh)
    keep_a, ap = _adv(advection, mesh)
    _check(lib().oracle_ac_diagonal(ctypes.byref(mesh), ctypes.byref(params), ctypes.byref(time), _dptr(lin),
                                    mp, ap, _dptr(d), threads or os.cpu_count()), "ac_diagonal")
    return d


def ch_blocks(mesh, params, time, lin, threads=0, mask=None, advection=None):
    C, N = params.n_grains + 2, n_nodes(mesh)
    lin = np.ascontiguousarray(lin, dtype=np.float64).reshape(C, N)
    b = np.zeros((4, N))
    keep, mp = _mptr(mask, mesh)
    keep_a, ap = _adv(advection, mesh)
    _check(lib().oracle_ch_blocks(ctypes.byref(mesh), ctypes.byref(params), ctypes.byref(time), _dptr(lin),
                                  mp, ap, _dptr(b), threads or os.cpu_count()), "ch_blocks")
    return b


def ch_matrix(mesh, params, time, lin, threads=0, mask=None, advection=None):
    """Assembled CH block, (3^dim, 4, N): 2x2 blocks per node row and neighbour."""
    C, N = params.n_grains + 2, n_nodes(mesh)
    NK = 27 if mesh.dim == 3 else 9
    lin = np.ascontiguousarray(lin, dtype=np.float64).reshape(C, N)
    A = np.zeros((NK, 4, N))
    keep, mp = _mptr(mask, mesh)
    keep_a, ap = _adv(advection, mesh)
    _check(lib().oracle_ch_matrix(ctypes.byref(mesh), ctypes.byref(params), ctypes.byref(time), _dptr(lin),
                                  mp, ap, _dptr(A), threads or os.cpu_count()), "ch_matrix")
    return A


def ch_sgs(mesh, A, r):
    """Multicolour symmetric Gauss-Seidel of the assembled CH block applied to r (2, N)."""
    N = n_nodes(mesh)
    A = np.ascontiguousarray(A, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(2, N)
    z = np.zeros((2, N))
    _check(lib().oracle_ch_sgs(ctypes.byref(mesh), _dptr(A), _dptr(r), _dptr(z)), "ch_sgs")
    return z


def inverse_diagonal(d):
    """operator_base.h:386-388: 1/d where |d| > 1e-10, else 1."""
    d = np.asarray(d, dtype=np.float64)
    return np.where(np.abs(d) > 1.0e-10, 1.0 / np.where(d == 0, 1.0, d), 1.0)


def grain_segments(mesh, eta, threshold_lower):
    """Particles of one order parameter (nodal values eta, length N): cell ids
    (int32 per cell, -1 = none) and the number of particles."""
    eta = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)
    ids = np.zeros(n_cells(mesh), dtype=np.int32)
    n = ctypes.c_int()
    _check(lib().oracle_grain_segments(ctypes.byref(mesh), _dptr(eta), float(threshold_lower),
                                       ids.ctypes.data_as(ctypes.POINTER(_c_int)), ctypes.byref(n)), "grain_segments")
    return ids, n.value


def segment_properties(mesh, eta, ids, n_particles, origin=(0.0, 0.0, 0.0)):
    """(n_particles, 3 + dim): measure, center, radius, max value per particle."""
    eta = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    org = np.ascontiguousarray(origin, dtype=np.float64)
    props = np.zeros((n_particles, 3 + mesh.dim))
    _check(lib().oracle_segment_properties(ctypes.byref(mesh), _dptr(org), _dptr(eta),
                                           ids.ctypes.data_as(ctypes.POINTER(_c_int)), int(n_particles),
                                           _dptr(props)), "segment_properties")
    return props


def advection_forces(mesh, params, u, cell_segments, centers, origin=(0.0, 0.0, 0.0), k=1.0, cgb=0.0, ceq=1.0,
                     smoothening=0.0, mask=None):
    """(n_segments, 1 + dim + (3 or 1)): volume, force, torque per segment
    (AdvectionOperatorGeneric::evaluate_forces)."""
    C, N = params.n_grains + 2, n_nodes(mesh)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(C, N)
    seg = np.ascontiguousarray(cell_segments, dtype=np.int32)
    cen = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
    org = np.ascontiguousarray(list(origin) + [0.0] * (3 - len(origin)), dtype=np.float64)
    nc = 1 + mesh.dim + (3 if mesh.dim == 3 else 1)
    out = np.zeros((cen.shape[0], nc))
    keep, mp = _mptr(mask, mesh)
    _check(lib().oracle_advection_forces(ctypes.byref(mesh), ctypes.byref(params), _dptr(org), _dptr(u), mp,
                                         seg.ctypes.data_as(ctypes.POINTER(_c_int)), _dptr(cen), cen.shape[0],
                                         float(k), float(cgb), float(ceq), float(smoothening), _dptr(out)),
           "advection_forces")
    return out


def advection_velocities(dim, vft, centers, mt, mr):
    """(n_segments, 9) velocity table (translation, angular velocity, center)
    from volumes, forces and torques (AdvectionMechanism)."""
    vft = np.ascontiguousarray(vft, dtype=np.float64)
    cen = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((cen.shape[0], 9))
    _check(lib().oracle_advection_velocities(int(dim), _dptr(vft), _dptr(cen), cen.shape[0], float(mt), float(mr),
                                             _dptr(out)), "advection_velocities")
    return out


def advection_courant(mesh, params, advection, dt, mask=None):
    """CFLChecker::check_courant: True when |v| dt < cell diameter everywhere."""
    keep, mp = _mptr(mask, mesh)
    keep_a, ap = _adv(advection, mesh)
    r = lib().oracle_advection_courant(ctypes.byref(mesh), ctypes.byref(params), mp, ap, float(dt))
    if r < 0:
        raise ValueError("advection_courant: bad arguments")
    return bool(r)


# --- periodic constraints (DoFTools::make_periodicity_constraints) ---------
# In a periodic direction d the nodes at coordinate n[d] are slaves of the
# nodes at 0; chains resolve to the node with all such coordinates at 0.
# Constrained operators (OperatorBase::vmult, operator_base.h:294-353) read
# masters for slaves, add the slave rows to the master rows and give the
# slave rows the identity (J v) or zero (residual).


def periodic_pairs(mesh, dirs):
    """(slave, master) node indices of the periodic directions `dirs`."""
    dim = mesh.dim
    nn = [mesh.n[d] + 1 for d in range(dim)]
    idx = np.arange(int(np.prod(nn)))
    co = [(idx // int(np.prod(nn[:d]))) % nn[d] for d in range(dim)]
    slave = np.zeros(idx.size, dtype=bool)
    mco = [c.copy() for c in co]
    for d in dirs:
        on = co[d] == mesh.n[d]
        slave |= on
        mco[d][on] = 0
    master = sum(mco[d] * int(np.prod(nn[:d])) for d in range(dim))
    return idx[slave], master[slave]


def periodic_resolve(mesh, u, dirs):
    sl, ma = periodic_pairs(mesh, dirs)
    out = np.array(u, dtype=np.float64, copy=True)
    out[:, sl] = out[:, ma]
    return out


def periodic_condense(mesh, dst, src, dirs, mode):
    """mode 0: slave rows = src (J v); 1: zero (residual); 2: the
    preconditioner outputs' identity (CH blocks 1, 0, 0, 1; AC diagonal 1)."""
    sl, ma = periodic_pairs(mesh, dirs)
    out = np.array(dst, dtype=np.float64, copy=True)
    for c in range(out.shape[0]):
        np.add.at(out[c], ma, dst[c, sl])
        if mode == 0:
            out[c, sl] = src[c, sl]
        elif mode == 1:
            out[c, sl] = 0.0
        else:
            out[c, sl] = 0.0 if c in (1, 2) else 1.0
    return out


def periodic_jvp(mesh, params, time, lin, src, dirs, **kw):
    C, N = params.n_grains + 2, n_nodes(mesh)
    src = np.asarray(src, dtype=np.float64).reshape(C, N)
    d = jvp(mesh, params, time, periodic_resolve(mesh, np.asarray(lin).reshape(C, N), dirs),
            periodic_resolve(mesh, src, dirs), **kw)
    return periodic_condense(mesh, d, src, dirs, 0)


def periodic_residual(mesh, params, time, u, hist, with_td, dirs, **kw):
    C, N = params.n_grains + 2, n_nodes(mesh)
    r = residual(mesh, params, time, periodic_resolve(mesh, np.asarray(u).reshape(C, N), dirs),
                 [periodic_resolve(mesh, np.asarray(h).reshape(C, N), dirs) for h in hist], with_td, **kw)
    return periodic_condense(mesh, r, None, dirs, 1)


def segment_periodicity(mesh, ids, dirs):
    """Distinct pairs (p, q), p <= q, of particles owning cells that face each
    other across the periodic boundaries `dirs` (tracker.h:1290-1336)."""
    dim = mesh.dim
    n = [mesh.n[d] for d in range(dim)]
    cells = np.asarray(ids).reshape(tuple(reversed(n)))  # (.., y, x)
    out = set()
    for d in dirs:
        ax = dim - 1 - d
        lo = np.take(cells, 0, axis=ax).ravel()
        hi = np.take(cells, n[d] - 1, axis=ax).ravel()
        for p, q in zip(lo, hi):
            if p >= 0 and q >= 0:
                out.add((int(min(p, q)), int(max(p, q))))
    return sorted(out)
