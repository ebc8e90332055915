"""Extract hpsint's golden test vectors for the sintering operator into JSON.

Run once with the path of an hpsint checkout as the only argument
(`python tests/golden/make_golden.py <path-to-hpsint>`); the JSON fixtures it
writes next to this script are committed, so nothing at test time reads the
reference tree.

Sources (paths inside the hpsint project):
  tests/residual_generic_{scalar,tensorial}_no_rbm.mpirun=1.output
      residual blocks of the 2x1-cell debug state, 4 significant digits
  tests/include/pf-applications/tests/sintering_model.h:53-239
      the model those residuals come from (parameters are re-typed below
      from lines 64-72 and 78-98 and cited, not parsed)
  applications/sintering/include/pf-applications/sintering/initial_values_debug.h:39-65
      nodal state of the 2D debug case
  tests/residual_generic_{scalar,tensorial}_rbm.mpirun=1.output
      the same residuals with the advection mechanism (rigid-body motion):
      tests/include/pf-applications/tests/sintering_model.h:74-76 (mt, mr),
      :119 (tracker threshold_lower), :214-217 (k, cgb, ceq, smoothening)
      are re-typed below, the residuals parsed
  tests/free_energy_sintering.{cc,output}
      known-answer values of the Wang free energy and its derivatives
  tests/power_sum.{cc,output}
      power sums
  tests/tangent_generic_{scalar,tensorial}.cc + .mpirun=1.output
      tolerances of the analytic-vs-finite-difference tangent check
  tests/grain_tracker_elliptical.{cc,mpirun=4.output}
      grain-tracker segments (center, radius, max value) of the spherical
      representation; the mesh, the indicator field and the threshold are
      re-typed below from the .cc (lines cited), the segments are parsed
  tests/grain_tracker_advection_periodic.{cc,mpirun=4.output}
      grains and their segments at t = 0 on a periodic mesh (a particle cut
      by the periodic boundary is one grain of two segments); the mesh, the
      particles, the interface width and the threshold are re-typed from the
      .cc, the segments are parsed
  tests/advection_mechanism_data.{cc,output}
      advection velocities (translation, rotation, total) of three grain
      segments at the cell barycenters of a 4 x 4 mesh; mt and mr are re-typed
      from the .cc, volumes/forces/torques/centers and velocities are parsed
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_residual(path):
    blocks = []
    lines = open(path).read().splitlines()
    for i, line in enumerate(lines):
        if line.startswith("Vector data:"):
            blocks.append([float(x) for x in lines[i + 1].split()])
    return blocks


def parse_free_energy(path):
    out = {}
    for line in open(path).read().splitlines():
        if not line.strip():
            break  # first section only; the other four repeat it
        m = re.match(r"^(\w+) = (\S+)$", line)
        if m:
            out[m.group(1)] = float(m.group(2))
    return out


def parse_power_sum(path):
    txt = open(path).read().splitlines()
    res = {"generalized": {}, "optimized": {}}
    section = None
    for line in txt:
        if line.startswith("Generalized"):
            section = "generalized"
        elif line.startswith("Optimized"):
            section = "optimized"
        elif line.startswith("std::array"):
            res[section]["input"] = [float(x) for x in line.split("=")[1].split()]
            res[section].setdefault("sums", {})
        m = re.match(r"^p=(\d+): (\S+)$", line)
        if m and "sums" in res[section]:
            res[section]["sums"].setdefault(m.group(1), float(m.group(2)))
    return res


def parse_tracker_segments(path, section):
    """Segments printed after the `section` header line (up to the next blank line)."""
    segs, on = [], False
    for line in open(path).read().splitlines():
        if line.startswith(section):
            on = True
            continue
        if on and not line.strip():
            break
        m = re.match(r"^\s+segment: center = (\S+) (\S+) \| radius = (\S+) \| max_value = (\S+)$", line)
        if on and m:
            segs.append([float(x) for x in m.groups()])
    return segs


def parse_tracker_grains(path, time_header):
    """Grains printed after `time_header`: [{"op": k, "segments": [[cx, cy,
    radius, max value], ...]}, ...] in the printed order."""
    grains, on = [], False
    for line in open(path).read().splitlines():
        if line.startswith("Time t = "):
            if on:
                break
            on = line.strip() == time_header
            continue
        if not on:
            continue
        m = re.match(r"^op_index_current = (\d+) \| op_index_old = \d+ \| segments = (\d+)$", line)
        if m:
            grains.append({"op": int(m.group(1)), "segments": []})
            continue
        m = re.match(r"^\s+segment: center = (\S+) (\S+) \| radius = (\S+) \| max_value = (\S+)$", line)
        if m:
            grains[-1]["segments"].append([float(x) for x in m.groups()])
    return grains


def parse_advection(path):
    """advection_mechanism_data output: the grain data and centers, then per
    cell batch and order parameter the velocities; deal.II prints a
    vectorized 2D tensor as x of both lanes, then y of both lanes."""
    out = {"batches": []}
    for line in open(path).read().splitlines():
        if line.startswith("grains_data:"):
            out["grains_data"] = [float(x) for x in line.split(":")[1].split()]
        elif line.startswith("grain_center:"):
            out["grain_center"] = [float(x) for x in line.split(":")[1].split()]
        elif line.startswith("cell_batch"):
            out["batches"].append([])
        else:
            m = re.match(r"^\s+op = (\d+) \| has_velocity = (\d) \| trans_vel = (.*) \| rot_vel = (.*) \| "
                         r"tot_vel = (.*)$", line)
            if m:
                out["batches"][-1].append({
                    "op": int(m.group(1)), "has_velocity": int(m.group(2)),
                    "trans_vel": [float(x) for x in m.group(3).split()],
                    "rot_vel": [float(x) for x in m.group(4).split()],
                    "tot_vel": [float(x) for x in m.group(5).split()]})
    return out


def main(ref):
    t = os.path.join(ref, "tests")
    golden = {
        "source": "hpsint tests (see make_golden.py for file list)",
        # sintering_model.h:64-72 and :78-98
        "model": {
            "dim": 2,
            "cells": [2, 1],
            "h": [1.0, 1.0],
            "A": 1.0, "B": 1.0, "kappa_c": 0.1, "kappa_p": 0.1,
            "Mvol": 1e-1, "Mvap": 1e-8, "Msurf": 1e1, "Mgb": 1e0, "L": 1e1,
            "bdf1_dt": 1e-5,
            "note": "old solution == current solution, so the BDF1 time term cancels",
        },
        # initial_values_debug.h:39-65: (x, y) -> (c, mu, eta1, eta2)
        "debug_state": {
            "0,0": [1.0, 0.1, 1.0, 0.0],
            "1,0": [0.8, 0.2, 0.4, 0.4],
            "2,0": [1.0, 0.3, 0.0, 1.0],
            "0,1": [1.0, 0.4, 1.0, 0.0],
            "1,1": [0.8, 0.5, 0.4, 0.4],
            "2,1": [1.0, 0.6, 0.0, 1.0],
        },
        # deal.II enumerates the DoFs of subdivided_hyper_rectangle cell by
        # cell: (0,0) (1,0) (0,1) (1,1) of cell 0, then (2,0) (2,1) of cell 1
        "dealii_dof_points": [[0, 0], [1, 0], [0, 1], [1, 1], [2, 0], [2, 1]],
        "residual_scalar": parse_residual(
            os.path.join(t, "residual_generic_scalar_no_rbm.mpirun=1.output")),
        "residual_tensorial": parse_residual(
            os.path.join(t, "residual_generic_tensorial_no_rbm.mpirun=1.output")),
        "residual_digits": 4,
        "residual_scalar_rbm": parse_residual(
            os.path.join(t, "residual_generic_scalar_rbm.mpirun=1.output")),
        "residual_tensorial_rbm": parse_residual(
            os.path.join(t, "residual_generic_tensorial_rbm.mpirun=1.output")),
        # sintering_model.h:74-76, :119, :214-217; segments are the tracker's
        # particles of each order parameter (threshold 1e-15)
        "rbm": {"k": 25.0, "cgb": 0.0, "ceq": 1.0, "smoothening": 0.0, "mt": 1.0, "mr": 1.0,
                "threshold_lower": 1e-15},
        # free_energy_sintering.cc: FreeEnergy(A=2, B=3), c=0.95, mu=0, etas
        "free_energy_kat": {
            "A": 2.0, "B": 3.0, "c": 0.95, "mu": 0.0,
            "etas": [0.3, 0.15, 0.47, 0.0],
            "values": parse_free_energy(os.path.join(t, "free_energy_sintering.output")),
            "digits": 6,
        },
        "power_sum": parse_power_sum(os.path.join(t, "power_sum.output")),
        # tangent_generic_scalar.cc / tangent_generic_tensorial.cc defaults,
        # and tangent_tester.h:38-106 (l1 norm of the difference, FD eps 1e-7
        # from lac/evaluation.h:30-87)
        "tangent": {
            "fd_epsilon": 1e-7,
            "scalar": {"tol_abs": 1e-3, "tol_rel": 1e-6},
            "tensorial": {"tol_abs": 1e0, "tol_rel": 1e-5},
            "outputs": {
                "scalar": open(os.path.join(t, "tangent_generic_scalar.mpirun=1.output")).read().splitlines()[0],
                "tensorial": open(os.path.join(t, "tangent_generic_tensorial.mpirun=1.output")).read().splitlines()[0],
            },
        },
    }
    # grain_tracker_elliptical.cc:56-60 (indicator of an ellipse and a circle,
    # interpolated at the nodes), :81-93 ([0, 9]^2, 10 x 10 subdivisions, 3
    # global refinements -> 80 x 80 cells), :124 (threshold_lower)
    golden["grain_tracker_spherical"] = {
        "mesh": {"dim": 2, "cells": [80, 80], "lower": [0.0, 0.0], "upper": [9.0, 9.0]},
        "ellipse": {"center": [4.0, 2.0], "semi_axes": [3.0, 1.0], "inclusive": True},
        "circle": {"center": [4.0, 6.5], "radius": 1.5, "inclusive": False},
        "threshold_lower": 1e-15,
        # [center x, center y, radius, max value], in the order printed
        "segments": parse_tracker_segments(os.path.join(t, "grain_tracker_elliptical.mpirun=4.output"),
                                           "Spherical grain representation"),
        "digits": 6,
    }
    # grain_tracker_advection_periodic.cc:111-127 ([0, 60] x [0, 22.5], 26 x 10
    # subdivisions, 3 global refinements -> 208 x 80 cells, periodic in x and
    # y, interface width 2), :161-166 (five particles of radius 7.5 on
    # y = 11.25; the ones at x = 0 and x = 60 are one particle across the
    # periodic boundary), :201 (threshold_lower); profile of
    # initial_values_spherical.h:51-75 (1 inside R - w/2, (1 + cos(pi (r - R +
    # w/2) / w)) / 2 across the interface, 0 outside); order parameters as
    # printed (particles at 0, 30, 60 on op 0, at 15, 45 on op 1)
    golden["grain_tracker_periodic"] = {
        "mesh": {"dim": 2, "cells": [208, 80], "lower": [0.0, 0.0], "upper": [60.0, 22.5]},
        "periodic": [0, 1],
        "particles": [[0.0, 11.25, 7.5, 0], [15.0, 11.25, 7.5, 1], [30.0, 11.25, 7.5, 0], [45.0, 11.25, 7.5, 1],
                      [60.0, 11.25, 7.5, 0]],
        "interface_width": 2.0,
        "threshold_lower": 1e-15,
        "grains": parse_tracker_grains(os.path.join(t, "grain_tracker_advection_periodic.mpirun=4.output"),
                                       "Time t = 0"),
        "digits": 6,
    }
    # advection_mechanism_data.cc:38-46 (2D, [0, 1]^2, 2 global refinements
    # -> 4 x 4 cells, 2 lanes per cell batch), :72-73 (mt, mr), :104-116 (one
    # segment per order parameter: volume 1 + (i + 1) i, force (1 + i, 0),
    # torque 1 + i, center (i, i)); the velocities are parsed
    adv = parse_advection(os.path.join(t, "advection_mechanism_data.output"))
    adv.update({"dim": 2, "cells": [4, 4], "h": [0.25, 0.25], "lanes": 2, "mt": 1.0, "mr": 1.0,
                "n_comp_volume_force_torque": 4, "digits": 6})
    golden["advection_mechanism_data"] = adv
    with open(os.path.join(HERE, "hpsint_goldens.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", os.path.join(HERE, "hpsint_goldens.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the hpsint checkout>")
    main(sys.argv[1])
