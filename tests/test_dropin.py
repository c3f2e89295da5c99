"""The drop-in end to end: the reference's own program set-up calling this
repository's library through the reference's solver entry point.

oracle/_ref/dropin_program (oracle/ref_program.cpp, built by oracle/build_ref.sh)
reads an XML deck in the reference's format through the reference's
preprocessor, builds the mesh, boundary conditions, initial solution and red
cell with the reference's classes, and calls
gpu_solver::General_Purpose_Solver_mk_i -- linked from
integration/Solver_gpu_lbfs.cpp over liblbfs_b200.so in place of the
reference's Solver_gpu.cu -- which writes the solution back into the
reference's Solution.  The same inputs, as the program dumps them before the
call, step through the reference's own kernels compiled for the host
(oracle/_ref/libref_lbfs.so, the order of Solver_gpu.cu:749-1021); the two
solutions agree within FP64_RTOL.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from helpers import FP64_RTOL, rel_err

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_lbfs as R  # noqa: E402

PROGRAM = os.path.join(ROOT, "oracle", "_ref", "dropin_program")
needs_program = pytest.mark.skipif(not (os.path.exists(PROGRAM) and R.available()),
                                   reason="oracle/_ref/dropin_program not built (oracle/build_ref.sh needs the "
                                          "reference sources and liblbfs_b200.so)")


def read_params(path):
    out = {}
    for line in open(path):
        k, v = line.split()
        out[k] = float(v)
    return out


def read_inputs(path, p):
    nc, nb, nn, nt, ns = (int(p[k]) for k in ("n_cells", "n_bc", "n_nodes", "n_tris", "n_springs"))
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.copy()
    d = {"state": take(np.float64, 4 * nc).reshape(4, nc), "rho_type": take(np.int32, nb),
         "vel_type": take(np.int32, nb), "bc_values": take(np.float64, 4 * nb).reshape(nb, 4),
         "tris": take(np.int32, 3 * nt).reshape(nt, 3), "springs": take(np.int32, 4 * ns).reshape(ns, 4),
         "xyz_stress_free": take(np.float64, 3 * nn).reshape(nn, 3), "xyz_initial": take(np.float64, 3 * nn).reshape(nn, 3)}
    assert off == len(raw)
    return d


def reference_run(p, d, steps):
    """The reference's kernels (host build) on the inputs the program passed to the solver."""
    mesh = R.RefMesh(p["X"], p["Y"], p["Z"], p["dt"], (p["origin_x"], p["origin_y"], p["origin_z"]), p["visc"])
    rp = R.RefParams()
    rp.visc, rp.delta_t, rp.gamma_inv, rp.channel_diameter = p["visc"], p["delta_t"], 1 / p["pre_conditioned_gamma"], p["Y"]
    rp.force[:] = (p["force_x"], p["force_y"], p["force_z"])
    rp.ref_rho, rp.max_velocity, rp.testcase = p["ref_rho"], p["max_velocity"], int(p["testcase"])
    rp.visc_factor_initial = 1.0 if int(p["testcase"]) == 2 else 0.0  # zero-filled managed memory before t = 1
    rp.has_rbc = 0 if int(p["testcase"]) == 2 else 1
    for k in ("volume_modulus", "local_area_modulus", "global_area_modulus", "shear_modulus", "global_bending_modulus",
              "local_bending_modulus", "membrane_thickness", "viscosity", "wlc_ratio", "curvature_ratio",
              "volume_ratio", "internal_viscosity_ratio", "reference_length"):
        setattr(rp, k, p[k])
    rp.pivkin_length, rp.sphere_reference = int(p["pivkin_length"]), int(p["sphere_reference"])
    rp.viscosity_period, rp.time_stepping = 10000, int(p["time_stepping"])
    rp.pre_conditioned_gamma, rp.preconditioning = p["pre_conditioned_gamma"], int(p["preconditioning"])
    rp.object_periodic = int(p["periodic"])
    rc = R.RefCase(mesh, rp, d["rho_type"], d["vel_type"], d["bc_values"])
    rc.set_state(*d["state"])
    if rp.has_rbc:
        rc.set_rbc(d["tris"], d["springs"], d["xyz_stress_free"], d["xyz_initial"])
    rc.step(steps)
    out = rc.state()
    rc.close()
    return out


@needs_program
def test_dropin_program_reads_the_deck_as_the_reference():
    """CPU: the program's dump of the solver's inputs (no solver call) -- mesh size, scalars as the
    reference's preprocessor forms them, the red cell from the Osay files."""
    import ref_deck
    with tempfile.TemporaryDirectory() as d:
        deck, state, info = ref_deck.shear_rbc_deck(d, n=16, steps=10, level=2, radius_cells=3.0)
        r = subprocess.run([PROGRAM, deck, os.path.join(d, "run"), state, "--dump-only"], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        p = read_params(os.path.join(d, "run_params.txt"))
        assert int(p["n_cells"]) == info["n_cells"] and int(p["n_nodes"]) == info["n_nodes"]
        assert abs(p["visc"] - info["visc"]) < 1e-15 and p["delta_t"] == 0.5 and p["force_x"] == 0.0
        assert abs(p["shear_modulus"] - info["shear_modulus"]) < 1e-15
        inp = read_inputs(os.path.join(d, "run_inputs.bin"), p)
        s0 = np.fromfile(state).reshape(4, -1)
        assert np.array_equal(inp["state"], s0)
        assert set(np.unique(inp["vel_type"])) == {2, 10}


@pytest.mark.gpu
@needs_program
@pytest.mark.parametrize("workload", ["shear_rbc16", "poiseuille12"])
def test_dropin_program_matches_reference_kernels(workload):
    import ref_deck
    steps = 10
    with tempfile.TemporaryDirectory() as d:
        if workload == "shear_rbc16":
            deck, state, info = ref_deck.shear_rbc_deck(d, n=16, steps=steps, level=2, radius_cells=3.0)
        else:
            deck, state, info = ref_deck.poiseuille_deck(d, n=12, steps=steps)
        r = subprocess.run([PROGRAM, deck, os.path.join(d, "run"), state], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr + open(os.path.join(d, "run_log.txt")).read()[-2000:]
        p = read_params(os.path.join(d, "run_params.txt"))
        inp = read_inputs(os.path.join(d, "run_inputs.bin"), p)
        got = np.fromfile(os.path.join(d, "run_state.bin")).reshape(4, -1)
        want = reference_run(p, inp, steps)
        for k in range(4):
            assert rel_err(got[k], want[k]) < FP64_RTOL, (k, rel_err(got[k], want[k]))
        assert not np.array_equal(got, inp["state"])  # the solver stepped


REF_GPU = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_program")


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(PROGRAM) and os.path.exists(REF_GPU)),
                    reason="oracle/_ref/ref_gpu_program or dropin_program not built")
@pytest.mark.parametrize("workload", ["shear_rbc16", "poiseuille12", "poiseuille12_tolerance"])
def test_reference_gpu_solver_matches_dropin(workload):
    """The reference's own GPU solver (Solver_gpu.cu and its kernels built for sm_100a) and the drop-in,
    each behind the same program set-up and deck, agree within FP64_RTOL after 10 steps.  With a
    tolerance in the deck (one no step meets) the drop-in runs its time loop through lbfs_step_until,
    the convergence test on the device after every step."""
    import ref_deck
    with tempfile.TemporaryDirectory() as d:
        if workload == "shear_rbc16":
            deck, state, _ = ref_deck.shear_rbc_deck(d, n=16, steps=10, level=2, radius_cells=3.0)
        elif workload == "poiseuille12":
            deck, state, _ = ref_deck.poiseuille_deck(d, n=12, steps=10)
        else:
            deck, state, _ = ref_deck.poiseuille_deck(d, n=12, steps=10, tolerance=1e-30)
        out = {}
        for name, prog in (("dropin", PROGRAM), ("reference", REF_GPU)):
            r = subprocess.run([prog, deck, os.path.join(d, name), state], capture_output=True, text=True,
                               timeout=600)
            assert r.returncode == 0, (name, r.stderr[-2000:])
            out[name] = np.fromfile(os.path.join(d, f"{name}_state.bin")).reshape(4, -1)
        for k in range(4):
            assert rel_err(out["dropin"][k], out["reference"][k]) < FP64_RTOL, (k, rel_err(out["dropin"][k],
                                                                                           out["reference"][k]))
