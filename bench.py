#!/usr/bin/env python
"""Benchmark of the LBFS-IBM time step on B200.

Workload (one GPU): wall-driven shear on an n^3-cell uniform hex mesh stored as
an unstructured face/cell list (default n = 64: 262,144 cells, 798,720 faces),
one red cell (level-3 icosphere: 642 nodes, 1,280 triangles, 1,920 springs,
radius 8 cells, capillary number 0.1) with the 4-point Peskin IBM delta, plain
FP64 -- the single-RBC shear configuration.  A "step" is one time step of the
solver.  hat2_value / hat2_e2e are the same workload on the reference's own
2-point hat stencil, the like-for-like counterpart of the reference arm.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: `value` is the device-timed throughput (Mcell-updates/s) with the
state resident in HBM, L2 flushed between timed steps (the 64^3 working set
fits in L2), each step timed by the library's CUDA events on its own streams;
`e2e` is the same metric through the C ABI with host buffers (page-locked H2D
of the state, the step, D2H of the state, every step); `roofline` is the
dominant kernel's algorithmic bytes per launch over its event-timed duration
against the measured HBM copy bandwidth; `cpu_baseline` is the reference's own
kernels compiled for the host (oracle/_ref) on a bounded sample.
Reference arm: the reference's own CPU implementation of the step (its kernel
sources compiled for the host, serial per instance) on every host core, one
instance per core.  For N > 1 GPUs each rank runs an independent replica of the
workload (the path has no exchange step between replicas): weak scaling.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))

METRIC = "Mcell-updates/s"
IBM_NAMES = {"peskin4": "4-point Peskin IBM", "hat2": "2-point hat IBM"}


def workload(n, n_cells, n_faces, n_nodes, n_tris, n_springs, ibm="peskin4"):
    """Name of the shear + red-cell workload at n^3 cells with its sizes."""
    return (f"shear_rbc: {n}^3-cell uniform hex mesh as unstructured faces ({n_cells} cells, {n_faces} faces), "
            f"wall shear (bc type 10), 1 red cell L3 icosphere ({n_nodes} nodes, {n_tris} triangles, "
            f"{n_springs} springs), radius 8 cells, Ca 0.1, {IBM_NAMES[ibm]}, FP64")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64, help="cells per axis")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-hat2", action="store_true", help="skip the run on the reference's 2-point hat stencil")
    ap.add_argument("--no-reference-programs", action="store_true",
                    help="reference arm: skip the reference's own GPU solver and CPU Solver programs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-ensemble section")
    ap.add_argument("--instances", type=int, default=64, help="instances of the batched ensemble")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint section")
    ap.add_argument("--no-precision", action="store_true", help="skip the jittered 128^3 FP32/FP64 precision study")
    ap.add_argument("--precision-steps", type=int, default=1000)
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--profile", type=int, default=0, metavar="STEPS",
                    help="profiling driver: build the --profile-case workload, run STEPS eager steps with flux_chunks 1 "
                         "(or --launch-shape) and exit without timing (a small case for ncu captures)")
    ap.add_argument("--profile-case", default="shear_rbc", choices=["shear_rbc", "jittered", "ensemble"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"], help="precision of the --profile run")
    ap.add_argument("--launch-shape", default=None,
                    help="JSON object of launch-shape fields to use instead of autotuning the headline workload "
                         "(e.g. the launch_shape a plain run printed, so a profiler run launches the same kernels)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def axis_geometry_uniform(mesh):
    """Whether every interior face of each axis has the same (area, dt, t1, t2), as the library
    checks at create (then the interior-face kernel takes the geometry from its parameters)."""
    import numpy as np
    if not getattr(mesh, "axis_aligned", True):
        return False
    ni, nfx, nfy = mesh.n_interior, mesh.n_face_x, mesh.n_face_y
    own, nb = np.asarray(mesh.owner)[:ni], np.asarray(mesh.neighbour)[:ni]
    cen, fc = np.asarray(mesh.cell_centroid).reshape(-1, 3), np.asarray(mesh.face_centroid).reshape(-1, 3)
    area, sdt = np.asarray(mesh.face_area)[:ni], np.asarray(mesh.streaming_dt)[:ni]
    for ax, (a, b) in enumerate(((0, nfx), (nfx, nfx + nfy), (nfx + nfy, ni))):
        if b <= a:
            continue
        t1 = cen[own[a:b], ax] - fc[a:b, ax]
        t2 = cen[nb[a:b], ax] - fc[a:b, ax]
        for v in (area[a:b], sdt[a:b], t1, t2):
            if not np.all(v == v[0]):
                return False
    return True


def ls_weights_coded(mesh):
    """Whether the folded least-squares weights W_q = LHS^-1 RHS_q of all cells take at most 8
    distinct vectors, as the library checks at create (then the gradient kernel reads a 3-bit code
    per stencil slot instead of the weights)."""
    import numpy as np
    L = np.asarray(mesh.lhs_inverse).reshape(-1, 3, 3)
    rh = np.asarray(mesh.rhs).reshape(-1, 6, 3)
    W = (L[:, None, :, 0] * rh[:, :, None, 0] + L[:, None, :, 1] * rh[:, :, None, 1]) + L[:, None, :, 2] * rh[:, :, None, 2]
    return len(np.unique(W.reshape(-1, 3), axis=0)) <= 8


def cell_update_closed_forms(mesh):
    """(faces, volume): whether the cell update forms each cell's six faces in closed form instead
    of reading its face list, and takes one 1 / volume from its parameters instead of one per cell,
    as the library checks at create.  The faces: an axis-aligned single mesh of the generator's
    structured layout (cell = i + nx (j + ny k)) whose face table -- per cell its faces in increasing
    order, +(f + 1) where it owns f, -(f + 1) where it is f's neighbour -- equals the closed form
    entry for entry.  The volume: every cell's 1 / volume the same, bit for bit."""
    import numpy as np
    inv = 1.0 / np.asarray(mesh.cell_volume, dtype=np.float64)[:mesh.n_cells]  # compared as the library does
    same_volume = bool(mesh.n_cells > 0 and np.all(inv == inv[0]))
    if not getattr(mesh, "axis_aligned", True) or mesh.delta_x <= 0:
        return False, same_volume
    q = [L / mesh.delta_x for L in (mesh.X, mesh.Y, mesh.Z)]
    n = [int(round(v)) for v in q]
    if any(m <= 0 or abs(v - m) >= 1e-9 * v for v, m in zip(q, n)):
        return False, same_volume
    nx, ny, nz = n
    nc, nf, ni = mesh.n_cells, mesh.n_faces, mesh.n_interior
    if nx * ny * nz != nc or (nx - 1) * ny * nz != mesh.n_face_x or nx * (ny - 1) * nz != mesh.n_face_y:
        return False, same_volume
    cells = np.concatenate([np.asarray(mesh.owner)[:nf], np.asarray(mesh.neighbour)[:ni]]).astype(np.int64)
    faces = np.concatenate([np.arange(nf), np.arange(ni)])
    signed = np.concatenate([np.arange(nf) + 1, -(np.arange(ni) + 1)])
    if cells.min() < 0 or cells.max() >= nc or np.any(np.bincount(cells, minlength=nc) != 6):
        return False, same_volume
    table = signed[np.lexsort((faces, cells))].reshape(nc, 6)
    c = np.arange(nc)
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    nfx, nfy, nfz = (nx - 1) * ny * nz, nx * (ny - 1) * nz, nx * ny * (nz - 1)
    bl = nfx + nfy + nfz
    br, bb = bl + ny * nz, bl + 2 * ny * nz
    bt, bk = bb + nx * nz, bb + 2 * nx * nz
    bf = bk + nx * ny
    f = np.stack([np.where(i > 0, (i - 1) + (nx - 1) * (j + ny * k), bl + j + ny * k),
                  np.where(i < nx - 1, i + (nx - 1) * (j + ny * k), br + j + ny * k),
                  np.where(j > 0, nfx + i + nx * ((j - 1) + (ny - 1) * k), bb + i + nx * k),
                  np.where(j < ny - 1, nfx + i + nx * (j + (ny - 1) * k), bt + i + nx * k),
                  np.where(k > 0, nfx + nfy + i + nx * (j + ny * (k - 1)), bk + i + nx * j),
                  np.where(k < nz - 1, nfx + nfy + i + nx * (j + ny * k), bf + i + nx * j)], axis=1)
    sg = np.stack([np.where(i > 0, -1, 1), np.ones(nc, np.int64), np.where(j > 0, -1, 1),
                   np.ones(nc, np.int64), np.where(k > 0, -1, 1), np.ones(nc, np.int64)], axis=1)
    o = np.argsort(f, axis=1, kind="stable")
    closed = np.take_along_axis(sg * (f + 1), o, axis=1)
    return bool(np.array_equal(table, closed)), same_volume


def algorithmic_bytes(mesh, phase, fp64=True):
    """Bytes each kernel must move once per launch (every array element it
    reads or writes counted once), FP64 storage."""
    nc, nf, ni, nb = mesh.n_cells, mesh.n_faces, mesh.n_interior, mesh.n_bc
    R = 8 if fp64 else 4
    if phase == "flux" and not getattr(mesh, "axis_aligned", True):
        # general-normal faces: per interior face ids 8, geometry (area, dt, n, t1, t2, branch) 12R,
        # flux out 4R; per bc face the same plus bc types/values 8 + 4R, bc record 9R, ghost state and
        # gradients out 16R; per cell: state 4R + 12 gradients 12R, visc factor R
        return ni * (8 + 16 * R) + nb * (16 + 45 * R) + nc * (17 * R)
    if phase == "flux":
        # per axis face: owner+neighbour ids 8, geometry (area, dt, t1, t2) 4R, flux out 4R;
        # per bc face: ids 8, geometry 12R, bc types/values 8 + 4R, bc record 9R, flux out 4R;
        # per cell: state 4R + 12 gradients 12R, visc factor R; per ghost: state and gradients out 16R.
        # On a mesh whose faces of each axis share one geometry the kernel reads it from its
        # parameters: no per-face geometry
        geo = 0 if axis_geometry_uniform(mesh) else 4 * R
        return ni * (8 + 4 * R + geo) + nb * (16 + 29 * R) + nc * (17 * R) + nb * (16 * R)
    if phase == "gradients":
        # per cell: stencil 24, folded weights 18R (or their 3-bit codes, 4, on a mesh with at most 8
        # distinct weight vectors), state 4R, gradients out 12R;
        # per ghost: bc record 9R + types 8 + values 4R (ghost states formed in registers)
        w = 4 if ls_weights_coded(mesh) else 18 * R
        return nc * (24 + 16 * R + w) + nb * (8 + 13 * R)
    if phase == "update":
        # per cell: face list 24, volume 8, t1 in/out 64, state out 4R; each face flux read once 4R.
        # The face list is formed in closed form on the generator's structured meshes, and one
        # 1 / volume comes from the parameters when every cell has it: neither is read then
        faces, volume = cell_update_closed_forms(mesh)
        return nc * ((0 if faces else 24) + (0 if volume else 8) + 64 + 4 * R) + nf * 4 * R
    return 0


def read_traffic(kernel, key):
    """DRAM bytes per launch of `kernel` on the workload `key` (e.g. shear_rbc_64_fp64) from the
    committed ncu summary profiles/dram_traffic.txt; None when that workload was not captured."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if line.startswith("#") or len(f) < 3 or f[0] != kernel or f[1] != key:
            continue
        try:
            return float(f[2])
        except ValueError:
            return None
    return None


_NOT_SHAPE = ("time_us", "step_us", "membrane_form_flushed_us", "source")  # printed beside the shape's fields


def tune_membrane_start(s, flush, reps=15):
    """The membrane chain's form (separate kernels or the cluster step) and start (beside K1 from the
    step's start, or behind K1's launch completion), chosen by timing flushed single graph steps as the
    timed region runs them; the library's autotuner times back-to-back steps with a warm L2, where the
    two regimes can prefer different forms.  Each candidate runs from a checkpoint of the same state,
    and the handle is restored to it afterwards.  Returns {(cluster, after): median us}."""
    import numpy as np
    import torch
    base = s.launch_shape()
    if not s.membranes:
        return {}
    blob = s.checkpoint()
    s.set_profiling(1)
    out = {}
    for cl in (0, 8, 16):
        for after in (0, 1):
            try:
                s.set_launch_shape(membrane_cluster=cl, membrane_after_k1=after)
            except Exception:  # a cluster the membranes do not fit
                continue
            s.restore(blob)
            s.step(2, graph=True)
            ts = []
            for k in range(reps):
                flush.fill_(k & 0xFF)
                torch.cuda.synchronize()
                s.step(1, graph=True)
                ts.append(s.phase_times()[5])
            out[(cl, after)] = 1e3 * float(np.median(ts))
    best = min(out, key=out.get)
    if out[best] < 0.99 * out[(base["membrane_cluster"], base["membrane_after_k1"])]:
        s.set_launch_shape(membrane_cluster=best[0], membrane_after_k1=best[1])
    else:
        s.set_launch_shape(membrane_cluster=base["membrane_cluster"], membrane_after_k1=base["membrane_after_k1"])
    s.restore(blob)
    return out


def velocity_errors(test, ref):
    """FP32-vs-FP64 velocity errors.  `field`: the velocity vector field's max-norm error relative to
    its largest magnitude, max_cells |u32 - u64| / max_cells |u64| (the relative field error the
    precision bound is stated in); `components`: each component's max error relative to that
    component's own largest magnitude (the cross-stream components of a shear flow are ~50x smaller
    than the stream velocity, so their FP32 storage noise floor is correspondingly higher)."""
    import numpy as np
    d = np.sqrt(sum((x - y) ** 2 for x, y in zip(test[1:], ref[1:])))
    mag = np.sqrt(sum(y ** 2 for y in ref[1:]))
    comps = {k: float(np.max(np.abs(x - y)) / np.max(np.abs(y))) for k, x, y in zip("uvw", test[1:], ref[1:])}
    return float(np.max(d) / np.max(mag)), comps


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_baseline_sample(n, budget_s=12.0, max_steps=200):
    """The reference's own kernels compiled for the host (oracle/_ref), serial,
    on the same workload with its 2-point IBM (the reference has no 4-point
    kernel); inputs from the reference's own generator (oracle/ref_cases.py)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lbfs
    if not ref_lbfs.available():
        return {"value": None, "unit": METRIC, "cores": 1, "kind": "reference",
                "sample": "oracle/_ref/libref_lbfs.so was not built"}
    import ref_cases
    solver, n_cells, _ = ref_cases.shear_rbc(n=n)
    solver.step(1)
    t0, steps = time.perf_counter(), 0
    while steps < max_steps and time.perf_counter() - t0 < budget_s:
        solver.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    solver.close()
    return {"value": n_cells * steps / dt / 1e6, "unit": METRIC, "cores": 1, "kind": "reference",
            "sample": f"{steps} steps of the {n}^3 + 1 red cell workload (2-point hat IBM), serial, {dt:.1f} s"}


def _ref_worker(args):
    """One reference instance: the workload built by the reference's own code
    (oracle/ref_cases.py) and stepped by its kernels compiled for the host; this
    process loads oracle/_ref/libref_lbfs.so and nothing of this repository's library."""
    n, steps, warmup = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_cases
    rc, n_cells, _ = ref_cases.shear_rbc(n=n)
    rc.step(warmup)
    t0 = time.perf_counter()
    rc.step(steps)
    dt = time.perf_counter() - t0
    rc.close()
    return n_cells * steps, dt


def _timed_program(program, make_deck, steps_pair, workdir, timeout=900):
    """Per-step host wall time of one of the reference's programs (oracle/ref_program.cpp behind the
    reference's set-up) from two runs of different step counts: the difference removes the set-up."""
    t = {}
    for n in steps_pair:
        d = os.path.join(workdir, f"{os.path.basename(program)}_{n}")
        deck, state, info = make_deck(d, n)
        r = subprocess.run([program, deck, os.path.join(d, "run"), state], capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"{os.path.basename(program)} exited {r.returncode}: {r.stderr[-300:]}")
        t[n] = float(open(os.path.join(d, "run_run.txt")).read().split()[1])
    n0, n1 = steps_pair
    per = (t[n1] - t[n0]) / (n1 - n0)
    return {"value": info["n_cells"] / per / 1e6, "unit": METRIC, "ms_per_step": per * 1e3,
            "timing": f"host wall clock of the solver call at {n1} and {n0} steps, difference over {n1 - n0} steps",
            "seconds": {str(k): v for k, v in t.items()}}


def reference_programs():
    """The reference's own GPU solver (Solver_gpu.cu and its kernels, unmodified, built for sm_100a with
    relocatable device code: oracle/_ref/ref_gpu_program) and its CPU Solver (oracle/_ref/ref_cpu_program),
    each behind the reference's program set-up reading an XML deck (oracle/ref_program.cpp,
    oracle/ref_deck.py): the 64^3 shear + L3 red cell workload (its 2-point IBM) and the 32^3 duct."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_deck
    gpu_prog = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_program")
    cpu_prog = os.path.join(ROOT, "oracle", "_ref", "ref_cpu_program")
    out = {}
    with tempfile.TemporaryDirectory(prefix="refprog") as work:
        shear = lambda d, n: ref_deck.shear_rbc_deck(d, n=64, steps=n, level=3, radius_cells=8.0)
        duct = lambda d, n: ref_deck.poiseuille_deck(d, n=32, steps=n)
        duct_cpu = lambda d, n: ref_deck.poiseuille_deck(d, n=32, steps=n, cpu_solver=True)
        if os.path.exists(gpu_prog):
            for name, mk, pair in (("shear_rbc64_hat2", shear, (50, 2050)), ("poiseuille32", duct, (50, 3050))):
                try:
                    out.setdefault("reference_gpu", {})[name] = _timed_program(gpu_prog, mk, pair, work)
                except Exception as exc:
                    out.setdefault("reference_gpu", {})[name] = {"value": None, "error": str(exc)}
            out["reference_gpu"]["what"] = ("the reference's Solver_gpu.cu time loop (every kernel followed by a "
                                            "device synchronize, managed memory) built for sm_100a, 1 B200")
        else:
            out["reference_gpu"] = {"unavailable": "oracle/_ref/ref_gpu_program was not built"}
        if os.path.exists(cpu_prog):
            try:
                out["reference_cpu_solver"] = dict(_timed_program(cpu_prog, duct_cpu, (3, 23), work), cores=1,
                                                   what="Solver::General_Purpose_Solver_mk_i (Solver.cpp:88-587), "
                                                        "serial, fluid only, on the 32^3 duct")
            except Exception as exc:
                out["reference_cpu_solver"] = {"value": None, "error": str(exc)}
    return out


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the step (its kernel sources
    compiled for the host, oracle/_ref), one serial instance per host core, on
    the benchmark workload with the reference's 2-point hat IBM (its uniform-mesh
    kernels have no 4-point delta).  Same warm-up and timed steps as the CUDA arm
    (steps capped at 200 so the run stays within minutes)."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lbfs
    if not ref_lbfs.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_lbfs.so was not built "
                          "(the reference sources were absent when build() ran)"}))
        return 0
    import multiprocessing as mp
    try:
        import psutil
        mem_procs = int(psutil.virtual_memory().available // (1200 * 2 ** 20))
    except Exception:
        mem_procs = os.cpu_count() or 1
    procs = max(1, min(os.cpu_count() or 1, mem_procs))
    steps = max(1, min(args.steps, 200))
    warmup = max(3, args.warmup)  # the CUDA arm's warm-up
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(args.n, steps, warmup)] * procs)
    wall = time.perf_counter() - t0
    cells = sum(r[0] for r in res)
    slowest = max(r[1] for r in res)
    value = cells / slowest / 1e6
    n = args.n
    nc = n ** 3
    nf = 3 * n * n * (n - 1) + 6 * n * n
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": slowest / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(n, nc, nf, 642, 1280, 1920, ibm="hat2"), "cells": nc, "faces": nf,
                   "membrane_nodes": 642, "ibm": "2-point hat",
                   "ibm_note": "the reference's uniform-mesh IBM kernels (immersed_boundary_method.cu:14-97, "
                               "947-1024) have only the 2-point hat stencil; the CUDA arm's headline uses the "
                               "4-point Peskin delta and reports the 2-point hat run as hat2_value / hat2_e2e",
                   "instances": procs, "parallelism": f"{procs} independent host processes, one instance each",
                   "inputs": "built by the reference's own generator and lagrangian_object (oracle/ref_cases.py); "
                             "no code of the CUDA arm is loaded"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "reference",
                         "sample": f"{steps} steps x {procs} instances of the {n}^3 workload, "
                                   f"reference kernels compiled for the host, one instance per core "
                                   f"(wall {wall:.1f} s incl. set-up)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_programs:
        line.update(reference_programs())
    print(json.dumps(line))
    return 0


def run_batched(args, K, warmup, flush, device, plain_fp64_value, rank=0, world=1):
    """Batched ensemble (independent shear channels of 16^3-48^3 cells with 1-8
    red cells each) in one handle, FP32 bulk and FP64, launch shapes autotuned;
    plus (one GPU) the same instances as separate handles, one graph each.  On
    N GPUs the instances are sharded by cost (cells + red-cell nodes, longest
    processing time first): each rank builds the ensemble of its own instances,
    nothing crosses ranks on the data path, and the aggregate throughput is all
    ranks' cells over the slowest rank's time (max over ranks)."""
    import dataclasses

    import numpy as np
    import torch

    from lbfs_b200 import GpuSolver, _abi, cases
    from lbfs_b200.parallel import gather_objects, max_over_ranks, shard_instances
    subset = None
    if world > 1:
        specs = cases.ensemble_specs(n_instances=args.instances)
        subset = shard_instances([sp["cost"] for sp in specs], world)[rank]
    ce = cases.ensemble(n_instances=args.instances, precision=_abi.LBFS_FP32_BULK, subset=subset)
    p64 = dataclasses.replace(ce.params, precision=_abi.LBFS_FP64)
    s32 = GpuSolver(ce.mesh, ce.params, ce.membranes, device=device)
    s64 = GpuSolver(ce.mesh, p64, ce.membranes, device=device)
    shapes = {}
    for name, x in (("fp32", s32), ("fp64", s64)):
        x.set_state(ce.rho, ce.u, ce.v, ce.w)
        x.step(1, graph=True)
        shapes[name] = x.autotune(reps=10)
        x.set_profiling(1)
        x.step(warmup - 1, graph=True)
    t = {"fp32": 0.0, "fp64": 0.0}
    for k in range(K):
        for name, x in (("fp32", s32), ("fp64", s64)):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            x.step(1, graph=True)
            t[name] += x.phase_times()[5]
    a, b = s64.state(), s32.state()
    err_field, err_comp = velocity_errors(b, a)
    drho = float(np.max(np.abs(b[0] - a[0])) / np.max(np.abs(a[0] - 1.0)))
    flags = (s32.status(), s64.status())
    launches = s32.launches_per_step()
    s32.close()
    s64.close()
    nc, nodes = ce.mesh.n_cells, ce.info["nodes"]
    members = ce.info["members"]
    if world > 1:
        # every rank: its shard's time; the job: all cells over the slowest rank
        per_rank = gather_objects({"rank": rank, "instances": len(members), "cells": nc,
                                   "value": nc * K / (t["fp32"] * 1e-3) / 1e6, "ms_per_step": t["fp32"] / K,
                                   "rel_err_velocity_vs_fp64": err_field})
        t_max = {k: max_over_ranks(v, device="cuda") for k, v in t.items()}
        cells_all = sum(r["cells"] for r in per_rank)
        val = {k: cells_all * K / (v * 1e-3) / 1e6 for k, v in t_max.items()}
        return {"value": val["fp32"], "unit": METRIC, "dtype": "f32 bulk (f64 reductions, node integration)",
                "instances": args.instances, "cells": cells_all, "n_gpus": world, "scaling": "strong",
                "sharding": "instances by cost (cells + red-cell nodes), longest processing time first; "
                            "no data-path collective", "per_rank": per_rank,
                "ms_per_step": t_max["fp32"] / K, "fp64_value": val["fp64"],
                "rel_err_velocity_vs_fp64": max(r["rel_err_velocity_vs_fp64"] for r in per_rank),
                "status_flags": flags, "launch_shape_fp32": shapes["fp32"]}
    val = {k: nc * K / (v * 1e-3) / 1e6 for k, v in t.items()}
    # the same instances as separate handles (one graph each, their own streams)
    Ks = min(K, 20)
    hs = []
    for m in members:
        h = GpuSolver(m.mesh, m.params, m.membranes, device=device)
        h.set_state(m.rho, m.u, m.v, m.w)
        h.step(warmup, graph=True)
        hs.append(h)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(Ks):
        for h in hs:
            h.step(1, graph=True)
    for h in hs:
        h.synchronize()
    sep = nc * Ks / (time.perf_counter() - t0) / 1e6
    for h in hs:
        h.close()
    return {"value": val["fp32"], "unit": METRIC, "dtype": "f32 bulk (f64 reductions, node integration)",
            "instances": len(members), "cells": nc, "faces": ce.mesh.n_faces, "membranes": ce.info["membranes"],
            "membrane_nodes": nodes, "ms_per_step": t["fp32"] / K, "rbc_node_steps_per_s": nodes * K / (t["fp32"] * 1e-3),
            "fp64_value": val["fp64"], "fp64_ms_per_step": t["fp64"] / K,
            "speedup_vs_plain_fp64": val["fp32"] / plain_fp64_value,
            "rel_err_velocity_vs_fp64": err_field, "rel_err_velocity_components_vs_fp64": err_comp,
            "rel_err_rho_deviation_vs_fp64": drho, "steps_compared": warmup + K, "status_flags": flags, "gpu_launches_per_step": launches,
            "launch_shape_fp32": shapes["fp32"], "launch_shape_fp64": shapes["fp64"],
            "separate_handles_fp32_value": sep,
            "separate_handles_timing": f"host wall clock over {Ks} steps of {len(members)} handles, one graph each",
            "workload": f"{len(members)} shear channels, n^3 cells with n uniform in [16, 48], 1-8 red cells "
                        "(level 2 or 3), G_s log-uniform in [2e-6, 2e-5], Ca uniform in [0.05, 0.5], "
                        "4-point Peskin IBM; seed 2024"}


def run_precision(args, device):
    """FP32-bulk vs FP64 precision study: 128^3 jittered hex mesh (interior
    vertices moved by up to 10 % of the spacing, general-normal fluxes on every
    face, faces' vector areas so that every cell closes), body-force duct flow
    with 16 L3 red cells, N steps in each precision; field and red-cell shape
    errors of the FP32 run against the FP64 run.  (With the reference
    importer's face areas the cells of this mesh do not close and the duct
    diverges in both precisions before 1000 steps.)"""
    import numpy as np

    from lbfs_b200 import GpuSolver, _abi, cases
    N = args.precision_steps
    out = {}
    runs = {}
    for name, prec in (("fp64", _abi.LBFS_FP64), ("fp32", _abi.LBFS_FP32_BULK)):
        c = cases.jittered_channel(precision=prec)
        with GpuSolver(c.mesh, c.params, c.membranes, device=device) as s:
            s.set_state(c.rho, c.u, c.v, c.w)
            s.step(3, graph=True)
            s.autotune(reps=5)
            s.set_profiling(1)
            t = 0.0
            for _ in range(N - 3):
                s.step(1, graph=True)
                t += s.phase_times()[5]
            runs[name] = (s.state(), s.nodes().reshape(-1, 3), s.status())
            out[name] = {"value": c.mesh.n_cells * (N - 3) / (t * 1e-3) / 1e6, "ms_per_step": t / (N - 3)}
            # per-kernel events on a few more steps (after the compared ones): K1, the general-normal
            # face fluxes (interior tiles + boundary faces beside them), K3 against the HBM peak
            s.set_profiling(2)
            s.step(2, graph=True)
            acc = np.zeros(6)
            for _ in range(10):
                s.step(1, graph=True)
                acc += s.phase_times()
            peaks, _ = measured_peaks()
            kr = {}
            for i, (ph, kn) in ((1, ("gradients", "k_cell_gradients")), (2, ("flux", "k_face_flux_general")),
                                (3, ("update", "k_cell_update"))):
                ms = acc[i] / 10
                b_ = algorithmic_bytes(c.mesh, ph, fp64=(name == "fp64"))
                kr[kn] = {"algorithmic_bytes": b_, "ms": ms, "achieved_gbs": b_ / (ms * 1e-3) / 1e9,
                          "frac": b_ / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"]}
            out[name]["kernel_roofline"] = kr
        info = c.info
    (r64, x64, f64), (r32, x32, f32) = runs["fp64"], runs["fp32"]
    rel_inf = {k: float(np.max(np.abs(a - b)) / np.max(np.abs(b))) for k, a, b in zip("uvw", r32[1:], r64[1:])}
    rel_l2 = {k: float(np.linalg.norm(a - b) / np.linalg.norm(b)) for k, a, b in zip("uvw", r32[1:], r64[1:])}
    R = info["radius_cells"] * 2.0
    return {"workload": f"128^3 jittered hex mesh (jitter 0.1 of the spacing, seed 1313; 2097152 cells, general-normal "
                        f"fluxes), body-force duct, {info['n_rbc']} L3 red cells radius 6 cells, 4-point Peskin IBM, "
                        f"{N} steps per precision",
            "fp64": out["fp64"], "fp32_bulk": out["fp32"], "speedup": out["fp32"]["value"] / out["fp64"]["value"],
            "rel_err_velocity_inf": rel_inf, "rel_err_velocity_l2": rel_l2,
            "rel_err_rho_deviation_inf": float(np.max(np.abs(r32[0] - r64[0])) / np.max(np.abs(r64[0] - 1.0))),
            "rbc_shape_err_over_radius": float(np.max(np.abs(x32 - x64)) / R),
            "status_flags": [f64, f32], "unit": METRIC}


def run_adjoint(args, device):
    """Discrete adjoint on the adjoint configuration: 48^3 shear channel, one
    level-4 red cell (2562 nodes, 5120 triangles, radius 8 cells), FP64,
    objective = Taylor deformation after N steps, checkpoints every 25 steps;
    gradient in the shear modulus, the bending modulus and the wall velocity,
    against central differences."""
    import dataclasses

    import numpy as np

    from lbfs_b200 import GpuSolver, cases
    c = cases.shear_rbc(n=48, level=4, radius_cells=8.0, rotate=True)
    c.membranes = [dataclasses.replace(m, internal_viscosity_ratio=1.0) for m in c.membranes]
    N, K = args.adjoint_steps, 25
    # plain forward step of the same case (graph, device events)
    with GpuSolver(c.mesh, c.params, c.membranes, device=device) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.set_profiling(1)
        s.step(5, graph=True)
        acc = 0.0
        for _ in range(50):
            s.step(1, graph=True)
            acc += s.phase_times()[5]
        fwd_ms = acc / 50
    with GpuSolver(c.mesh, c.params, c.membranes, device=device) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        J, g, t = s.adjoint(N, K, membrane=0)
    # the same with every segment recomputed from its checkpoint in the reverse sweep
    os.environ["LBFS_ADJOINT_MEMORY_MB"] = "0"
    try:
        with GpuSolver(c.mesh, c.params, c.membranes, device=device) as s:
            s.set_state(c.rho, c.u, c.v, c.w)
            J_rr, g_rr, t_rr = s.adjoint(N, K, membrane=0)
    finally:
        del os.environ["LBFS_ADJOINT_MEMORY_MB"]

    def taylor(gs=1.0, kb=1.0, su=1.0):
        mems = [dataclasses.replace(m, shear_modulus=m.shear_modulus * gs,
                                    global_bending_modulus=m.global_bending_modulus * kb) for m in c.membranes]
        bcv = c.mesh.bc_values
        keep = bcv.copy()
        bcv[:, :3] *= su
        try:
            with GpuSolver(c.mesh, c.params, mems, device=device) as s:
                s.set_state(c.rho, c.u, c.v, c.w)
                s.step(N, graph=True)
                xyz = s.nodes().reshape(-1, 3)
        finally:
            bcv[:] = keep
        dx, dy = xyz[:, 0] - xyz[:, 0].mean(), xyz[:, 1] - xyz[:, 1].mean()
        Ixx, Iyy, Ixy = np.sum(dx * dx), np.sum(dy * dy), np.sum(dx * dy)
        T, D = 0.5 * (Ixx + Iyy), 0.5 * (Ixx - Iyy)
        R = np.sqrt(D * D + Ixy * Ixy)
        L, B = np.sqrt(T + R), np.sqrt(T - R)
        return (L - B) / (L + B)

    m = c.membranes[0]
    scale = {"shear_modulus": m.shear_modulus, "bending_modulus": m.global_bending_modulus,
             "velocity_scale": 1.0}
    fd = {}
    for h in (1e-6, 1e-4):
        fd[h] = {"shear_modulus": (taylor(gs=1 + h) - taylor(gs=1 - h)) / (2 * h * scale["shear_modulus"]),
                 "bending_modulus": (taylor(kb=1 + h) - taylor(kb=1 - h)) / (2 * h * scale["bending_modulus"]),
                 "velocity_scale": (taylor(su=1 + h) - taylor(su=1 - h)) / (2 * h)}
    rel = {h: {k: abs(g[k] - v) / abs(v) if v != 0 else None for k, v in d.items()} for h, d in fd.items()}
    # the finite-difference noise floor of the wall-velocity derivative: its effect on J over the window is
    # small, so central differences at small h sit in the rounding of J; sweep h and report the
    # difference quotient's error against the adjoint at each h, with J's change at that h
    j0 = taylor()
    sweep = {}
    for h in (1e-7, 1e-6, 1e-5, 1e-4, 1e-3):
        jp, jm = taylor(su=1 + h), taylor(su=1 - h)
        q = (jp - jm) / (2 * h)
        sweep[f"{h:g}"] = {"fd": q, "rel_err_vs_adjoint": abs(g["velocity_scale"] - q) / abs(q) if q != 0 else None,
                           "delta_J_over_J": abs(jp - jm) / abs(j0), "J_rounding_over_J": 2.2e-16 * 50}
    return {"workload": "48^3 shear channel (110592 cells), 1 red cell L4 icosphere (2562 nodes, 5120 triangles), "
                        f"radius 8 cells, Ca 0.1, 4-point Peskin IBM, FP64, {N} steps, checkpoint every {K}",
            "objective": "Taylor deformation (L - B)/(L + B) of the red cell in the x-y plane at the final step",
            "J": J, "gradient": g,
            "gradient_note": "d/d shear modulus, d/d bending modulus, d/d sigma with every wall velocity value x sigma",
            "forward_ms_per_step": fwd_ms, "adjoint_forward_sweep_ms": t[0], "adjoint_reverse_sweep_ms": t[1],
            "reverse_over_forward": t[1] / (N * fwd_ms),
            "total_over_forward": (t[0] + t[1]) / (N * fwd_ms),
            "reverse_over_forward_note": "reverse sweep per step over one plain forward step (graph, device events); "
                                         "the trajectory's intermediates (about 8 GB here) fit in half the free "
                                         "device memory, so the forward sweep keeps them and the reverse sweep "
                                         "recomputes nothing; total_over_forward counts both sweeps",
            "recompute": {"adjoint_forward_sweep_ms": t_rr[0], "adjoint_reverse_sweep_ms": t_rr[1],
                          "reverse_over_forward": t_rr[1] / (N * fwd_ms),
                          "total_over_forward": (t_rr[0] + t_rr[1]) / (N * fwd_ms),
                          "same_results": bool(J_rr == J and g_rr == g),
                          "note": "LBFS_ADJOINT_MEMORY_MB=0: checkpoints only, every segment recomputed in the "
                                  "reverse sweep"},
            "fd_h1e-6": fd[1e-6], "rel_err_h1e-6": rel[1e-6], "fd_h1e-4": fd[1e-4], "rel_err_h1e-4": rel[1e-4],
            "velocity_fd_sweep": sweep,
            "velocity_fd_sweep_note": "central differences of J in the wall-velocity scale at relative steps h; "
                                      "J_rounding_over_J is an estimate of J's own rounding (50 ulp), the floor "
                                      "below which delta_J_over_J carries no digits"}


def run_profile(args):
    """A few eager steps of one workload and nothing else: the program ncu captures."""
    from lbfs_b200 import GpuSolver, _abi, cases
    prec = _abi.LBFS_FP32_BULK if args.precision == "fp32" else _abi.LBFS_FP64
    if args.profile_case == "jittered":
        c = cases.jittered_channel(n=args.n, precision=prec)
    elif args.profile_case == "ensemble":
        c = cases.ensemble(n_instances=args.instances, precision=prec)
    else:
        c = cases.shear_rbc(n=args.n, precision=prec)
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        if args.launch_shape:
            s.set_launch_shape(**{k: v for k, v in json.loads(args.launch_shape).items() if k not in _NOT_SHAPE})
        else:
            s.set_launch_shape(flux_chunks=1)
        s.step(args.profile)
        s.synchronize()
        print(json.dumps({"profile": args.profile_case, "n": args.n, "precision": args.precision, "steps": args.profile,
                          "status_flags": s.status(), "launch_shape": s.launch_shape()}))
    return 0


def main():
    from lbfs_b200.parallel import dist_env, max_over_ranks
    args = parse()
    rank, local_rank, world = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.profile:
        return run_profile(args)
    import numpy as np
    import torch
    import torch.distributed as dist
    import ctypes
    from datetime import timedelta

    from lbfs_b200 import GpuSolver, _abi, cases

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local_rank))
    warmup = max(3, args.warmup)
    K = args.steps
    c = cases.shear_rbc(n=args.n)
    mesh = c.mesh
    n_nodes = sum(m.n_nodes for m in c.membranes)
    n_tris = sum(len(m.tris) for m in c.membranes)
    n_springs = sum(len(m.springs) for m in c.membranes)
    s = GpuSolver(mesh, c.params, c.membranes, device=local_rank)
    s.set_state(c.rho, c.u, c.v, c.w)
    flush = torch.empty(512 * 2 ** 20, dtype=torch.uint8, device="cuda")  # 512 MB > 126 MB L2
    s.step(warmup, graph=True)
    if args.launch_shape:
        fixed = {k: v for k, v in json.loads(args.launch_shape).items() if k not in _NOT_SHAPE}
        s.set_launch_shape(**fixed)
        shape = dict(s.launch_shape(), source="--launch-shape")
    else:
        shape = s.autotune(reps=40)  # launch shape by whole-step timing (the library's autotuner)
        flushed = tune_membrane_start(s, flush)
        shape = dict(s.launch_shape(), step_us=shape["step_us"],
                     membrane_form_flushed_us={f"cluster{k[0]}_after{k[1]}": round(v, 1) for k, v in flushed.items()})
    s.set_profiling(1)  # events around each whole step only
    s.step(2, graph=True)
    s.synchronize()
    launches_per_step = s.launches_per_step()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_pass():
        acc = np.zeros(6)
        for k in range(K):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            s.step(1, graph=True)
            acc += s.phase_times()  # synchronises the solver stream; outside the events
        return acc

    sampler = ClockSampler(local_rank)
    barrier()
    sampler.start()
    step_sum = timed_pass()
    barrier()
    clocks = sampler.stop()
    t_step_ms = step_sum[5] / K
    total_s = max_over_ranks(step_sum[5] / 1e3, device="cuda")
    cell_updates = mesh.n_cells * K * world
    value = cell_updates / total_s / 1e6
    # second timed pass with per-kernel events (they cost a few us per step, so
    # the headline above is timed without them).  The kernels run one after the
    # other here (no chunk pipelining of K1 -> K2), so each event pair times one
    # kernel and not its overlap with another; the membrane chain still overlaps.
    chosen_chunks = s.launch_shape()["flux_chunks"]
    s.set_launch_shape(flux_chunks=1)
    s.set_profiling(2)
    s.step(2, graph=True)
    phase_sum = timed_pass()
    s.set_profiling(1)
    s.set_launch_shape(flux_chunks=chosen_chunks)
    phases = {name: phase_sum[i] / K for i, name in enumerate(["membrane", "gradients", "flux", "update"])}
    status = s.status()

    # roofline of the dominant fluid kernel (the membrane kernel overlaps them on a second stream)
    fluid = {k: v for k, v in phases.items() if k != "membrane"}
    dom = max(fluid, key=fluid.get)
    peaks, peak_kind = measured_peaks()
    alg = algorithmic_bytes(mesh, dom)
    achieved = alg / (fluid[dom] * 1e-3) / 1e9
    kname = {"flux": "k_face_flux", "gradients": "k_cell_gradients", "update": "k_cell_update"}[dom]
    traffic = read_traffic(kname, f"shear_rbc_{args.n}_fp64")
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": alg, "launch_ms": fluid[dom],
                "timing": "per-kernel CUDA events, second timed pass of K steps with K1 and K2 not pipelined"}
    # every fluid kernel against the same HBM peak (algorithmic bytes / event-timed duration)
    kernel_roofline = {}
    for ph, kn in (("gradients", "k_cell_gradients"), ("flux", "k_face_flux"), ("update", "k_cell_update")):
        b_ = algorithmic_bytes(mesh, ph)
        gbs = b_ / (fluid[ph] * 1e-3) / 1e9
        kernel_roofline[kn] = {"algorithmic_bytes": b_, "ms": fluid[ph], "achieved_gbs": gbs,
                               "frac": gbs / peaks["hbm_gbs"],
                               "traffic": read_traffic(kn, f"shear_rbc_{args.n}_fp64")}

    def e2e_pass(h):
        """End to end through the C ABI with page-locked host buffers: every step the
        state goes host -> device, the step runs, the state comes back."""
        n = mesh.n_cells
        host = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
        for hh, a in zip(host, h.state()):
            hh[:] = a
        h.set_profiling(False)
        Ke = min(K, 50)
        barrier()
        t0 = time.perf_counter()
        for _ in range(Ke):
            _abi.check(_abi.lib().lbfs_set_state(h._h, *[_abi.ptr(x) for x in host]))
            h.step(1, graph=True)
            _abi.check(_abi.lib().lbfs_get_state(h._h, *[_abi.ptr(x) for x in host]))
        barrier()
        te = max_over_ranks(time.perf_counter() - t0, device="cuda")
        return {"value": n * Ke * world / te / 1e6, "unit": METRIC, "h2d_bytes_per_step": 4 * 8 * n,
                "d2h_bytes_per_step": 4 * 8 * n, "steps": Ke, "timing": "host wall clock around set_state, step, "
                "get_state (page-locked host arrays)"}

    def e2e_run(h, steps=100):
        """End to end the way the reference's own loop uses its solver (Solver_gpu.cu's time loop
        behind General_Purpose_Solver_mk_i): the state host -> device once, every step followed by
        the device -> host read of its residual norms (the convergence check), the state back once;
        host wall clock over the whole call, page-locked host arrays."""
        n = mesh.n_cells
        host = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
        for hh, a in zip(host, h.state()):
            hh[:] = a
        h.set_profiling(False)
        res = torch.empty(4, dtype=torch.float64, pin_memory=True).numpy()
        barrier()
        t0 = time.perf_counter()
        _abi.check(_abi.lib().lbfs_set_state(h._h, *[_abi.ptr(x) for x in host]))
        for _ in range(steps):
            h.step(1, graph=True)
            _abi.check(_abi.lib().lbfs_get_residuals(h._h, _abi.ptr(res)))
        _abi.check(_abi.lib().lbfs_get_state(h._h, *[_abi.ptr(x) for x in host]))
        barrier()
        te = max_over_ranks(time.perf_counter() - t0, device="cuda")
        return {"value": n * steps * world / te / 1e6, "unit": METRIC, "h2d_bytes_per_step": 4 * 8 * n / steps,
                "d2h_bytes_per_step": 4 * 8 * n / steps + 4 * 8, "steps": steps,
                "timing": "host wall clock around set_state, then per step step + get_residuals (4 doubles), "
                          "then get_state (page-locked host arrays)"}

    def e2e_device_loop(h, steps=100):
        """The reference's loop through lbfs_step_until: the state host -> device once, the steps with
        the convergence test of every step on the device (a CUDA graph while node; tolerance 0, so all
        `steps` run), the last residual norms and the state back once; host wall clock."""
        n = mesh.n_cells
        host = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
        for hh, a in zip(host, h.state()):
            hh[:] = a
        h.set_profiling(False)
        h.step_until(2, 0.0)  # the loop graph built outside the timed region
        res = torch.empty(4, dtype=torch.float64, pin_memory=True).numpy()
        done = ctypes.c_int32()
        barrier()
        t0 = time.perf_counter()
        _abi.check(_abi.lib().lbfs_set_state(h._h, *[_abi.ptr(x) for x in host]))
        _abi.check(_abi.lib().lbfs_step_until(h._h, steps, 0.0, ctypes.byref(done), _abi.ptr(res)))
        _abi.check(_abi.lib().lbfs_get_state(h._h, *[_abi.ptr(x) for x in host]))
        barrier()
        te = max_over_ranks(time.perf_counter() - t0, device="cuda")
        assert done.value == steps
        return {"value": n * steps * world / te / 1e6, "unit": METRIC, "h2d_bytes_per_step": 4 * 8 * n / steps,
                "d2h_bytes_per_step": (4 * 8 * n + 4 * 8) / steps, "steps": steps,
                "timing": "host wall clock around set_state, lbfs_step_until (convergence test on the device "
                          "after every step), get_state (page-locked host arrays)"}

    e2e = None if args.no_e2e else e2e_pass(s)
    e2e_reference_loop = None if args.no_e2e else e2e_run(s)
    e2e_device_loop_value = None if args.no_e2e else e2e_device_loop(s)

    # the same workload on the reference's own IBM stencil (2-point hat): the like-for-like
    # counterpart of the reference arm, which has no 4-point kernel
    hat2 = None
    if not args.no_hat2:
        ch = cases.shear_rbc(n=args.n, ibm_stencil=_abi.LBFS_IBM_HAT2)
        sh = GpuSolver(ch.mesh, ch.params, ch.membranes, device=local_rank)
        sh.set_state(ch.rho, ch.u, ch.v, ch.w)
        sh.step(warmup, graph=True)
        sh.autotune(reps=40)
        tune_membrane_start(sh, flush)
        sh.set_profiling(1)
        sh.step(2, graph=True)
        acc = 0.0
        barrier()
        for k in range(K):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            sh.step(1, graph=True)
            acc += sh.phase_times()[5]
        barrier()
        th = max_over_ranks(acc / 1e3, device="cuda")
        hat2 = {"value": mesh.n_cells * K * world / th / 1e6, "ms_per_step": acc / K,
                "e2e": None if args.no_e2e else e2e_pass(sh),
                "e2e_reference_loop": None if args.no_e2e else e2e_run(sh),
                "e2e_device_loop": None if args.no_e2e else e2e_device_loop(sh), "status_flags": sh.status(),
                "workload": workload(args.n, mesh.n_cells, mesh.n_faces, n_nodes, n_tris, n_springs, ibm="hat2")}
        sh.close()

    # FP32-bulk form on the same workload: throughput and field error against this FP64 run
    # the sections below describe the forms on one GPU; a multi-GPU run reports the replicas and the sharded ensemble
    fp32 = None
    if rank == 0 and world == 1:
        c32 = cases.shear_rbc(n=args.n, precision=_abi.LBFS_FP32_BULK)
        c64 = cases.shear_rbc(n=args.n)
        a, b = GpuSolver(mesh, c64.params, c64.membranes, device=local_rank), \
            GpuSolver(c32.mesh, c32.params, c32.membranes, device=local_rank)
        for x in (a, b):
            x.set_state(c.rho, c.u, c.v, c.w)
            x.step(2, graph=True)
            x.autotune(reps=40)
            tune_membrane_start(x, flush)
            x.set_profiling(1)
        b.step(warmup, graph=True)
        a.step(warmup, graph=True)
        tb = 0.0
        for k in range(K):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            b.step(1, graph=True)
            tb += b.phase_times()[5]
            a.step(1, graph=True)
        sa, sb = a.state(), b.state()
        err_field, err_comp = velocity_errors(sb, sa)
        drho = float(np.max(np.abs(sb[0] - sa[0])) / np.max(np.abs(sa[0] - 1.0)))
        fp32 = {"value": mesh.n_cells * K / (tb * 1e-3) / 1e6, "unit": METRIC, "speedup_vs_fp64": None,
                "rel_err_velocity_vs_fp64": err_field, "rel_err_velocity_components_vs_fp64": err_comp,
                "rel_err_rho_deviation_vs_fp64": drho,
                "steps_compared": warmup + K}
        fp32["speedup_vs_fp64"] = fp32["value"] / (mesh.n_cells * K / (step_sum[5] * 1e-3) / 1e6)
        a.close()
        b.close()

    batched = None
    if not args.no_batched:
        # on N GPUs every rank takes its shard of the instances (the collectives inside are taken by all ranks)
        batched = run_batched(args, K, warmup, flush, local_rank, mesh.n_cells * K / (step_sum[5] * 1e-3) / 1e6,
                              rank, world)

    precision = None
    if rank == 0 and world == 1 and not args.no_precision:
        try:
            precision = run_precision(args, local_rank)
        except Exception as exc:
            precision = {"error": f"{type(exc).__name__}: {exc}"}

    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        try:
            adjoint = run_adjoint(args, local_rank)
        except Exception as exc:
            adjoint = {"error": f"{type(exc).__name__}: {exc}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_sample(args.n)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": 1, "kind": "reference", "sample": f"failed: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K, "warmup": warmup,
            "ms_per_step": t_step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.n, mesh.n_cells, mesh.n_faces, n_nodes, n_tris, n_springs),
                       "cells": mesh.n_cells, "faces": mesh.n_faces, "membrane_nodes": n_nodes, "ibm": "4-point Peskin",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "flushed between timed steps (512 MB write)", "graph": "CUDA graph per step"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "e2e_reference_loop": e2e_reference_loop, "e2e_device_loop": e2e_device_loop_value,
            "gpu_launches": launches_per_step * K,
            "launch_shape": shape,
            "clocks": clocks,
            "kernel_ms": phases,
            "kernel_roofline": kernel_roofline,
            "rbc_node_steps_per_s": n_nodes * K * world / total_s,
            "hat2_value": None if hat2 is None else hat2["value"],
            "hat2_e2e": None if hat2 is None else hat2["e2e"],
            "hat2": hat2,
            "fp32_bulk": fp32,
            "batched": batched,
            "adjoint": adjoint,
            "precision_study": precision,
            "status_flags": status,
        }
        print(json.dumps(line))
    s.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
