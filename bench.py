#!/usr/bin/env python
"""DTFE interpolation throughput on B200: grid samples/s.

Workload (default): 256^3 Zel'dovich-displaced particles (rms displacement
1.0 lattice spacing, velocities 100 km/s per unit displacement + N(0, 50
km/s)) in a periodic 100 Mpc/h box, interpolated to a 256^3 grid.  A step is
one pass of the hot path over the resident tessellation: vertex densities
(FP64 volume reduction), seed bins, then one fused walk+interpolation launch
producing cell-centre density, velocity, velocity gradient, divergence,
shear and vorticity for every cell.  A grid sample is one fully evaluated
output cell.  The host tessellation is built once before timing (the
reference's CGAL step, excluded from the metric as it is cached).

Keys beyond the base contract:
  e2e          the same metric through the C ABI with host buffers: every step
               uploads the tessellation and vertex data from pinned memory and
               copies all output fields back
  roofline     k_interpolate against the measured HBM copy bandwidth
  cpu_baseline the CPU oracle (restated reference path) on the host cores,
               on a bounded sample of the same workload
  mc           Monte-Carlo cell average (8 points per cell) throughput

--impl reference times the reference's CPU path (the oracle port: no CGAL or
Boost exists here to build the reference itself) with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
          "velocity_vorticity"]
C_OUT = 1 + 3 + 9 + 1 + 5 + 3  # output floats per cell
METRIC = "grid samples/s DTFE dens+vel-grad 256^3 vs plain GPU & CPU at ≤1e-5 rel; bwd/fwd"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="particles per side (and grid cells per side)")
    ap.add_argument("--threads", type=int, default=0, help="host threads (0 = all)")
    ap.add_argument("--e2e-steps", type=int, default=9)
    ap.add_argument("--e2e-buffers", type=int, default=3,
                    help="handles used in turn by the end-to-end loop (2 = double buffering)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mc", action="store_true")
    ap.add_argument("--no-m1", action="store_true")
    ap.add_argument("--variants", default="", help="locate,eval launch variants (default: autotune)")
    ap.add_argument("--m1-points", type=int, default=100, help="method-1 points per cell (reference default 100)")
    ap.add_argument("--bwd-n", type=int, default=128, help="particles per side of the backward workload")
    ap.add_argument("--no-bwd", action="store_true")
    ap.add_argument("--fd-particles", type=int, default=1000)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=10)
    ap.add_argument("--sampling-n", type=int, default=128,
                    help="particles per side of the redshift-cone / user-point workload (one box)")
    ap.add_argument("--no-sampling", action="store_true")
    ap.add_argument("--no-output", action="store_true", help="skip the binary output-file leg")
    ap.add_argument("--no-tess", action="store_true", help="skip the GPU tessellation leg")
    ap.add_argument("--scalars", type=int, default=0,
                    help="extra N(0,1) scalar fields per particle, interpolated with their gradients")
    ap.add_argument("--fp64-cells", type=int, default=50000,
                    help="cells checked against the FP64 oracle in the CPU-baseline leg (0 = none)")
    ap.add_argument("--split", action="store_true",
                    help="split one box over the ranks (the reference's sub-boxes dealt to ranks, tiles "
                         "gathered to rank 0 every step: strong scaling) instead of one box per rank")
    ap.add_argument("--cpu-kind", default="auto", choices=["auto", "port"],
                    help="CPU baseline: the reference's code when built (auto) or the oracle port")
    return ap.parse_args()


def host_threads(req: int) -> int:
    if req > 0:
        return req
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def tessellation_leg(plan) -> dict:
    """The Delaunay tessellations of the step's padded sub-box point sets on
    the GPU (dtfe_gpu_tessellate, CUDA events around the call) beside the host
    tessellator's time for the same sets (host_prep_s.tessellation_s), and
    whether every set's tetrahedra equal the host's array for array."""
    from dtfe_b200 import device as D
    sets = [plan.xyz[b.vert_offset:b.vert_offset + b.n_verts] for b in plan.boxes]
    D.tessellate([sets[0][:64]])  # module load, small allocations
    out, ms, why = D.tessellate(sets, return_ms=True, return_stats=True)
    equal = []
    for b, (tv, st) in zip(plan.boxes, out):
        host = plan.tet_v[b.tet_offset:b.tet_offset + b.n_tets] - np.int32(b.vert_offset)
        equal.append(bool(st == 0 and tv.shape == host.shape and np.array_equal(tv, host)))
    return {"gpu_ms": ms, "host_s": plan.timings.get("tessellation_s"), "sets": len(sets),
            "vertices": int(sum(len(x) for x in sets)), "tetrahedra": int(sum(len(tv) for tv, _ in out)),
            "equal_to_host": all(equal), "sets_equal": int(sum(equal)),
            "status": [st for _, st in out if st], "failed_stars": {k: v for k, v in why.items() if v > 0}}


def build_workload(n: int, rank: int, threads: int, scalars: int = 0):
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    t0 = time.time()
    pos, psi = S.zeldovich_lattice(n, S.BOX, 1.0, seed=1 + 1000 * rank)
    rng = np.random.default_rng(2 + 1000 * rank)
    vel = (100.0 * psi / (S.BOX / n) + rng.normal(0.0, 50.0, psi.shape)).astype(np.float32)
    del psi
    w = np.ones(len(pos), np.float32)
    sc = (np.random.default_rng(8 + 1000 * rank).standard_normal((len(pos), scalars)).astype(np.float32)
          if scalars else None)
    t_ics = time.time() - t0
    t0 = time.time()
    plan = P.make_plan(pos, w, vel, sc, grid=(n, n, n), n_threads=threads,
                       average_density_value=float(len(pos)) / S.BOX ** 3)
    plan.timings["ics_s"] = t_ics
    plan.timings["plan_total_s"] = time.time() - t0
    # the input particles, for the upload that ships them once
    plan.particles = {"pos": pos, "weight": w, "velocity": vel, "scalar": sc}
    return plan


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per k_interpolate launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "interp_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def workload_config(args, plan, world: int) -> dict:
    """The workload block of the JSON line, the same for both arms."""
    return {"workload": f"zeldovich{args.n}: {args.n}^3 Zel'dovich particles (rms 1.0 spacing, "
                        f"periodic 100 Mpc/h, padding 5) -> {args.n}^3 grid, cell-centre "
                        "density+velocity+gradient+div/shear/vort"
                        + (f" + {args.scalars} N(0,1) scalars and their gradients" if args.scalars else "")
                        + " per step, vertex densities included",
            "grid": list(plan.grid), "particles": args.n ** 3, "vertices": plan.n_verts,
            "tetrahedra": plan.n_tets, "subboxes": plan.n_boxes,
            "l2": "inputs larger than L2 (tessellation arrays > 126 MB)",
            "parallelism": f"dp{world} (independent boxes per GPU)"}


def reference_code_step(plan, threads: int):
    """The reference's own code on the host cores, when the harness built
    from its sources is present (oracle/_ref): per sub-box, one host thread
    runs vertexDensity + interpolateGrid (density, velocity, velocity
    gradient; src/CGAL_triangulation/triangulation.cpp, unaveraged_interpolation.cc)
    as DTFE_parallel's OpenMP threads do, then DTFE()'s serial
    computeDivergenceShearVorticity on the main grid (src/DTFE.cpp:248-249):
    the same 22 floats per cell as the GPU step.  The step time is the
    slowest thread's plus the derived pass.  Returns (seconds, per-box
    seconds) or None."""
    import refharness as R
    if not R.available():
        return None
    return R.time_boxes(plan, threads, with_derived=os.path.exists(R.MAIN_LIB))


def reference_method1(plan, threads: int, n_points: int):
    """The reference's own vertexDensity + interpolateGrid_averaged_1 on all
    sub-boxes, one host thread each (the harness; None without it)."""
    try:
        import refharness as R
    except ImportError:
        return None
    if not R.available():
        return None
    t, per_box = R.time_boxes(plan, threads, which=1, n_points=n_points)
    G = int(np.prod(plan.grid))
    return {"cells_per_s": G / t, "cores": min(threads, plan.n_boxes), "kind": "reference",
            "step_s": t, "sample": f"the whole workload, {plan.n_boxes} sub-boxes on one host thread each; "
                                   f"sub-boxes {min(per_box):.2f}-{max(per_box):.2f} s"}


def fp64_check(plan, outs: dict, fields, cells: int, d32, d64) -> dict:
    """Error of the device's fields against the FP64 oracle on a sample:
    `cells` grid cells drawn uniformly from every sub-box's tile, evaluated
    by the oracle (FP64 mode, the sub-box's own tessellation) at the same
    float cell centres.  Per field: max |gpu - fp64| / max(|fp64|, rms(fp64))
    over the sample (the relative error with the field's RMS as the floor of
    the denominator), and the plain relative error max |gpu - fp64| / |fp64|
    over the entries with |fp64| above 1% of the field's RMS."""
    import torch
    import oracle as O
    rng = np.random.default_rng(123)
    G1, G2 = plan.grid[1], plan.grid[2]
    per_box = max(1, cells // plan.n_boxes)
    got = {f: [] for f in fields}
    want = {f: [] for f in fields}
    big = [-1e30, 1e30, -1e30, 1e30, -1e30, 1e30]
    for b in range(plan.n_boxes):
        B = plan.boxes[b]
        dims = [int(B.tile_dims[a]) for a in range(3)]
        if min(dims) <= 0:
            continue
        ijk = np.stack([rng.integers(0, dims[a], per_box) for a in range(3)], 1)
        pts = np.stack([plan.xs[B.coord_offset[0] + ijk[:, 0]], plan.ys[B.coord_offset[1] + ijk[:, 1]],
                        plan.zs[B.coord_offset[2] + ijk[:, 2]]], 1).astype(np.float32)
        cell = ((B.tile_origin[0] + ijk[:, 0]) * G1 + (B.tile_origin[1] + ijk[:, 1])) * G2 + (B.tile_origin[2]
                                                                                          + ijk[:, 2])
        ref = O.interpolate_points(plan, d32, d64, fields, pts, big, mode=O.MODE_FP64, box=b)
        sel = torch.from_numpy(cell.astype(np.int64)).to(next(iter(outs.values())).device)
        for f in fields:
            got[f].append(outs[f].index_select(0, sel).cpu().numpy().reshape(len(cell), -1))
            want[f].append(ref[f].reshape(len(cell), -1))
    err, plain = {}, {}
    for f in fields:
        a = np.concatenate(got[f]).astype(np.float64)
        w = np.concatenate(want[f])
        floor = max(np.sqrt(np.mean(w ** 2)), 1e-300)
        err[f] = float(np.max(np.abs(a - w) / np.maximum(np.abs(w), floor)))
        keep = np.abs(w) > 0.01 * floor
        plain[f] = float(np.max(np.abs(a[keep] - w[keep]) / np.abs(w[keep]))) if keep.any() else 0.0
    return {"cells": int(sum(len(x) for x in got[fields[0]])), "max_rel_err_rms_floor": err,
            "max_rel_err_plain_above_1pct_rms": plain, "max_over_fields": max(err.values()), "bar": 1e-5}


def cpu_baseline(plan, threads: int, target_s: float, kind: str = "auto", check=None) -> dict:
    """The reference's own code on the host cores (reference_code_step) on
    the whole workload; without the harness, the CPU oracle in the
    reference's arithmetic on a sample (vertex densities over the whole
    tessellation plus cell-centre interpolation of the first x-slabs of
    sub-box 0, scaled to the full grid)."""
    G = int(np.prod(plan.grid))
    import oracle as O
    ref = reference_code_step(plan, threads) if kind == "auto" else None
    if ref is not None:
        t, per_box = ref
        res = {"value": G / t, "unit": "grid samples/s", "cores": min(threads, plan.n_boxes), "kind": "reference",
               "sample": f"the whole workload: the reference's vertexDensity + interpolateGrid (density, velocity, "
                         f"velocity gradient) on all {plan.n_boxes} sub-boxes, one host thread each (its "
                         f"DTFE_parallel split), then its computeDivergenceShearVorticity on the main grid; "
                         f"step {t:.2f} s, sub-boxes {min(per_box):.2f}-{max(per_box):.2f} s",
               "step_s": t}
        if check is not None:
            d32, d64, _ = O.vertex_density(plan)
            res["fp64_check"] = fp64_check(plan, *check, d32, d64)
        return res
    import copy
    from dtfe_b200 import _native as N
    t0 = time.time()
    d32, d64, _ = O.vertex_density(plan)
    t_vd = time.time() - t0
    b0 = plan.boxes[0]
    per_slab = int(b0.tile_dims[1]) * int(b0.tile_dims[2])
    # calibrate: one slab, then enough slabs for the target time
    sub = copy.copy(plan)
    boxes = (N.Subbox * 1)()
    boxes[0] = b0
    sub.boxes = boxes
    slabs = 1
    elapsed = 0.0
    for _ in range(4):
        boxes[0].tile_dims[0] = slabs
        t0 = time.time()
        O.interpolate(sub, d32, d64, FIELDS, mode=O.MODE_REF, nthreads=threads)
        elapsed = time.time() - t0
        if elapsed > 0.25 * target_s or slabs >= int(b0.tile_dims[0]):
            break
        slabs = min(int(b0.tile_dims[0]), max(slabs * 2, int(slabs * target_s / max(elapsed, 1e-3))))
    cells = slabs * per_slab
    G = int(np.prod(plan.grid))
    t_step = t_vd + elapsed * G / cells
    res = {"value": G / t_step, "unit": "grid samples/s", "cores": threads, "kind": "port",
           "sample": f"vertex densities of all {plan.n_verts} vertices ({t_vd:.2f} s) + cell-centre "
                     f"interpolation of {cells} of {G} cells ({elapsed:.2f} s, x-slabs of sub-box 0), "
                     f"scaled to the full grid",
           "vertex_density_s": t_vd, "interp_cells_per_s": cells / elapsed}
    if check is not None:
        res["fp64_check"] = fp64_check(plan, *check, d32, d64)
    return res


def _events(stream, fn, steps):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def backward_leg(args, local: int, threads: int) -> dict:
    """Differentiation workload: 128^3 Zel'dovich particles (rms 0.5 spacing,
    weights U[0.5, 1.5], velocities as the main workload) -> 128^3 grid.
    Loss = sum a*density + b*divergence (DTFE) + sum a_cic*CIC + a_tsc*TSC
    with seeded N(0, 1) weights.  Forward: vertex densities + cell-centre
    density and divergence, CIC and TSC deposits; backward: the adjoints.
    Gradients of 1000 random particles are checked against FP64 central
    differences (h = 1e-6 box) of the oracle's loss."""
    import torch
    import oracle as O
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    from dtfe_b200.device import DeviceDTFE
    n = args.bwd_n
    cuda = torch.device("cuda", local)
    pos, psi = S.zeldovich_lattice(n, S.BOX, 0.5, seed=17)
    rng = np.random.default_rng(18)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (100.0 * psi / (S.BOX / n) + rng.normal(0.0, 50.0, psi.shape)).astype(np.float32)
    del psi
    avg = float(w.sum()) / S.BOX ** 3
    t0 = time.time()
    plan = P.make_plan(pos, w, vel, None, grid=(n, n, n), n_threads=threads, average_density_value=avg)
    dplans = {k: P.make_deposit_plan(pos, w, None, grid=(n, n, n), n_threads=threads, kind=k,
                                     average_density_value=avg) for k in ("CIC", "TSC")}
    t_plan = time.time() - t0
    G = int(np.prod(plan.grid))
    V = plan.n_verts
    a = torch.tensor(rng.standard_normal(G), dtype=torch.float32, device=cuda)
    b = torch.tensor(rng.standard_normal(G), dtype=torch.float32, device=cuda)
    ad = {k: torch.tensor(rng.standard_normal(G), dtype=torch.float32, device=cuda) for k in dplans}
    dens = torch.empty(G, device=cuda)
    div = torch.empty(G, device=cuda)
    dd = {k: torch.empty(G, device=cuda) for k in dplans}
    gx, gv, gw = (torch.empty((V, 3), device=cuda), torch.empty((V, 3), device=cuda), torch.empty(V, device=cuda))
    dgx = {k: torch.empty((d.n, 3), device=cuda) for k, d in dplans.items()}
    dgw = {k: torch.empty(d.n, device=cuda) for k, d in dplans.items()}
    dev = DeviceDTFE(local)
    ddev = {k: DeviceDTFE(local) for k in dplans}
    dev.load(plan)
    stream = torch.cuda.ExternalStream(dev.stream, device=cuda)
    torch.cuda.synchronize()

    def fwd():
        dev.vertex_density(plan.rho_bar)
        dev.interpolate_dev(["density", "velocity_divergence"], {"density": dens, "velocity_divergence": div})

    def bwd():
        dev.adjoint_dev(gx, grad_density=a, grad_divergence=b, grad_vel=gv, grad_w=gw)

    for _ in range(3):
        fwd()
        bwd()
    t_fwd = _events(stream, fwd, 5)
    t_bwd = _events(stream, bwd, 5)
    dep = {}
    for k, d in dplans.items():
        ds = torch.cuda.ExternalStream(ddev[k].stream, device=cuda)

        def dfwd():
            ddev[k].deposit_dev(d, dd[k])

        def dbwd():
            ddev[k].deposit_adjoint_dev(ad[k], dgx[k], dgw[k])
        for _ in range(3):
            dfwd()
            dbwd()
        dep[k] = {"fwd_ms": 1e3 * _events(ds, dfwd, 5), "bwd_ms": 1e3 * _events(ds, dbwd, 5),
                  "particle_copies": d.n}
    # finite-difference check on random particles
    sel = np.random.default_rng(19).choice(len(pos), min(args.fd_particles, len(pos)), replace=False)
    t0 = time.time()
    d32, d64, _ = O.vertex_density(plan)
    _, loc = O.interpolate(plan, d32, d64, ["density"], mode=O.MODE_FP64, want_loc=True, nthreads=threads)
    prob = O.AdjointProblem(plan, loc, a=a.cpu().numpy().astype(np.float64), b=b.cpu().numpy().astype(np.float64))
    fd = O.dtfe_fd(prob, plan.xyz, plan.weight, plan.velocity, sel, h_pos=1e-6 * S.BOX)

    def per_particle(src, g):
        out = np.zeros((len(pos),) + g.shape[1:])
        np.add.at(out, src, g.astype(np.float64))
        return out[sel]

    def rel(x, y):
        rms = max(float(np.sqrt(np.mean(y * y))), 1e-300)
        return float(np.max(np.abs(x - y) / np.maximum(np.abs(y), rms)))
    fd_err = {"dtfe_pos": rel(per_particle(plan.src, gx.cpu().numpy()), fd[:, :3]),
              "dtfe_vel": rel(per_particle(plan.src, gv.cpu().numpy()), fd[:, 3:6]),
              "dtfe_weight": rel(per_particle(plan.src, gw.cpu().numpy()), fd[:, 6])}
    for k, d in dplans.items():
        at = ad[k].cpu().numpy().astype(np.float64).reshape(plan.grid)
        fdx = np.zeros((len(sel), 3))
        fdw = np.zeros(len(sel))
        order = np.argsort(d.src, kind="stable")
        ss = d.src[order]
        offs = np.array([bx.particle_offset for bx in d.boxes] + [d.n])
        keep = np.ones(len(sel), bool)
        for r, i in enumerate(sel):
            for c in order[np.searchsorted(ss, i, "left"):np.searchsorted(ss, i, "right")]:
                bi = int(np.searchsorted(offs, c, "right") - 1)
                bx = d.boxes[bi]
                dims = np.array([bx.tile_dims[q] for q in range(3)], np.int32)
                org = [bx.tile_origin[q] for q in range(3)]
                if d.kind == 1:
                    # CIC weights have a kink at cell centres and the clipped edge
                    # stencils jump at cell faces: a central difference that
                    # straddles one is not a derivative, so such particles are left out
                    lo = np.array([bx.region[0], bx.region[2], bx.region[4]], np.float64)
                    dx = (np.array([bx.region[1], bx.region[3], bx.region[5]], np.float64) - lo) / dims
                    fr = (d.pos[c].astype(np.float64) - lo) / dx
                    fr -= np.floor(fr)
                    if np.min(np.minimum(np.abs(fr - 0.5), np.minimum(fr, 1 - fr)) * dx) < 4e-6 * S.BOX:
                        keep[r] = False
                ta = np.ascontiguousarray(at[org[0]:org[0] + dims[0], org[1]:org[1] + dims[1],
                                             org[2]:org[2] + dims[2]]).ravel()
                reg = np.array(list(bx.region), np.float32)
                h = 1e-6 * S.BOX
                for q in range(3):
                    pp, pm = d.pos[c:c + 1].astype(np.float64).copy(), d.pos[c:c + 1].astype(np.float64).copy()
                    pp[0, q] += h
                    pm[0, q] -= h
                    lp = O.deposit_loss_grad(d.kind, pp, d.weight[c:c + 1], reg, dims, d.rho_bar, ta, False)[0]
                    lm = O.deposit_loss_grad(d.kind, pm, d.weight[c:c + 1], reg, dims, d.rho_bar, ta, False)[0]
                    fdx[r, q] += (lp - lm) / (2 * h)
                fdw[r] += O.deposit_loss_grad(d.kind, d.pos[c:c + 1], np.ones(1), reg, dims, d.rho_bar, ta,
                                              False)[0]
        fd_err[f"{k.lower()}_pos"] = rel(per_particle(d.src, dgx[k].cpu().numpy())[keep], fdx[keep])
        fd_err[f"{k.lower()}_weight"] = rel(per_particle(d.src, dgw[k].cpu().numpy()), fdw)
        fd_err[f"{k.lower()}_pos_excluded_at_kinks"] = int((~keep).sum())
    t_fd = time.time() - t0
    dev.close()
    for d in ddev.values():
        d.close()
    return {"workload": f"zeldovich{n}: {n}^3 particles (rms 0.5 spacing, weights U[0.5,1.5]) -> {n}^3 grid; "
                        "loss = sum N(0,1)-weighted density + divergence grids (DTFE), CIC and TSC densities",
            "dtfe_fwd_ms": 1e3 * t_fwd, "dtfe_bwd_ms": 1e3 * t_bwd, "bwd_over_fwd": t_bwd / t_fwd,
            "deposit": dep,
            "deposit_note": "deposit forward includes the host->device copy of the particles (host-input API)",
            "fd_check": {"particles": int(len(sel)), "h": 1e-6 * S.BOX, "max_rel_err_rms_floor": fd_err,
                         "seconds": t_fd},
            "vertices": V, "tetrahedra": plan.n_tets, "host_plan_s": t_plan}


def compare_leg(args, plan, local: int, threads: int, cpu: bool = False) -> dict:
    """The comparison estimators on the main workload, device-timed: SPH with
    32 neighbours on the same padded sub-box particle sets and grid tiles,
    CIC and TSC deposition (their own paddings, the reference's sub-box
    split) of density and velocity.  With cpu (and the reference harness
    built), each also times the reference's own implementation on a sample
    of the same sub-boxes, one per host thread."""
    ref = None
    if cpu:
        import refharness as R
        ref = R if R.available() else None
    hthreads = host_threads(args.threads)
    import torch
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    from dtfe_b200.device import DeviceDTFE
    cuda = torch.device("cuda", local)
    G = int(np.prod(plan.grid))
    res = {}
    dev = DeviceDTFE(local)
    dev.load(plan)
    stream = torch.cuda.ExternalStream(dev.stream, device=cuda)
    d = torch.empty(G, device=cuda)
    v = torch.empty((G, 3), device=cuda)

    def sph():
        dev.sph_dev(plan.rho_bar, d, v, n_neighbors=32)
    sph()
    t = _events(stream, sph, 2)
    res["SPH32"] = {"ms": 1e3 * t, "grid_samples_per_s": G / t}
    dev.close()
    if ref is not None:
        rate, m = ref.time_sph_boxes(plan, hthreads, 32)
        res["SPH32"]["reference_cpu"] = {"grid_samples_per_s": rate, "boxes_sampled": m, "cores": min(m, hthreads),
                                         "kind": "reference", "sample": f"{m} of {plan.n_boxes} padded sub-boxes, "
                                                                         "one per host thread, density + velocity"}
    n = args.n
    pos, psi = S.zeldovich_lattice(n, S.BOX, 1.0, seed=1)
    rng = np.random.default_rng(2)
    vel = (100.0 * psi / (S.BOX / n) + rng.normal(0.0, 50.0, psi.shape)).astype(np.float32)
    del psi
    w = np.ones(len(pos), np.float32)
    for kind in ("CIC", "TSC"):
        dp = P.make_deposit_plan(pos, w, vel, grid=plan.grid, n_threads=threads, kind=kind,
                                 average_density_value=float(len(pos)) / S.BOX ** 3)
        # particle arrays in pinned host memory, as a caller streaming them would keep them
        for f in ("pos", "weight", "velocity"):
            a = getattr(dp, f)
            t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
            t.numpy()[...] = a
            setattr(dp, f, t.numpy())
        dd = DeviceDTFE(local)
        ds = torch.cuda.ExternalStream(dd.stream, device=cuda)

        def dep():
            dd.deposit_dev(dp, d, v)
        dep()
        t = _events(ds, dep, 3)
        # the same deposit with the particles already resident on the device
        pd, wd, vd = (torch.from_numpy(a).to(cuda) for a in (dp.pos, dp.weight, dp.velocity))
        torch.cuda.synchronize()

        def dep_resident():
            dd.deposit_resident(dp, pd, wd, vd, d, v)
        dep_resident()
        tr = _events(ds, dep_resident, 3)
        res[kind] = {"ms": 1e3 * tr, "grid_samples_per_s": G / tr, "particle_copies": dp.n,
                     "particles_per_s": dp.n / tr,
                     "note": "particles resident on the device (dtfe_gpu_deposit_resident)",
                     "host_input": {"ms": 1e3 * t, "grid_samples_per_s": G / t,
                                    "h2d_bytes": int(dp.pos.nbytes + dp.weight.nbytes + dp.velocity.nbytes),
                                    "note": "dtfe_gpu_deposit_dev: includes the host->device copy of the "
                                            "particles from pinned memory"}}
        del pd, wd, vd
        dd.close()
        if ref is not None:
            rate, m, npart = ref.time_deposit_boxes(dp, hthreads)
            res[kind]["reference_cpu"] = {"grid_samples_per_s": rate, "boxes_sampled": m, "cores": min(m, hthreads),
                                          "kind": "reference",
                                          "sample": f"{m} of {len(dp.boxes)} sub-box regions ({npart} particles), "
                                                    "one per host thread, density + velocity"}
    return res


def batch_leg(args, local: int, threads: int) -> dict:
    """Batched sub-boxes: 64 periodic sub-boxes (side 25 Mpc/h) with
    log-normal particle counts in [1e4, 1e6] (median 1e5), each a Zel'dovich
    lattice plus an NFW cluster (20% of its particles, r_s = 0.05 side),
    padding 10% of the side, each interpolated to its own 64^3 grid (density
    + velocity).  A step: vertex densities + seeds + interpolation of all 64
    tiles.  Timed three ways on the device: the captured CUDA graph replayed
    back to back, the same step through the C ABI calls, and one handle and
    launch sequence per sub-box (the unbatched loop)."""
    import torch
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    from dtfe_b200.device import DeviceDTFE
    cuda = torch.device("cuda", local)
    t0 = time.time()
    wl = S.workload("subboxes64_nfw")
    plan = P.make_subbox_plan(wl["subboxes"], grid=wl["grid"], padding_fraction=wl["padding_fraction"])
    t_plan = time.time() - t0
    fields = ["density", "velocity"]
    G = int(np.prod(plan.grid))
    outs = {"density": torch.empty((G, 1), device=cuda), "velocity": torch.empty((G, 3), device=cuda)}
    dev = DeviceDTFE(local)
    dev.load(plan)
    stream = torch.cuda.ExternalStream(dev.stream, device=cuda)
    dev.vertex_density(plan.rho_bar)
    variants = dev.autotune(fields)

    def plain():
        dev.vertex_density(plan.rho_bar)
        dev.interpolate_dev(fields, outs)
    for _ in range(3):
        plain()
    t_plain = _events(stream, plain, args.batch_steps)
    dev.graph_build(plan.rho_bar, fields, outs)
    for _ in range(3):
        dev.graph_launch()
    dev.synchronize()
    t_graph = _events(stream, dev.graph_launch, args.batch_steps)
    st = dev.read_status()
    # unbatched: one handle per sub-box, launches one sub-box at a time
    parts = P.split_boxes(plan)
    devs, pouts = [], []
    for p in parts:
        d = DeviceDTFE(local)
        d.load(p)
        d.set_variants(*variants)
        g = int(np.prod(p.grid))
        devs.append(d)
        pouts.append({"density": torch.empty((g, 1), device=cuda), "velocity": torch.empty((g, 3), device=cuda)})

    def loop():
        for d, o, p in zip(devs, pouts, parts):
            d.vertex_density(p.rho_bar)
            d.interpolate_dev(fields, o)
    for _ in range(2):
        loop()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        loop()
    torch.cuda.synchronize()
    t_loop = (time.perf_counter() - t0) / 3
    for d in devs:
        d.close()
    counts = [int(b.n_verts) for b in plan.box_list()]
    dev.close()
    return {"workload": "subboxes64_nfw: 64 periodic sub-boxes (side 25), log-normal counts in [1e4, 1e6] "
                        "(median 1e5), lattice + NFW cluster, padding 10%, 64^3 grid each, density + velocity",
            "grid_samples_per_step": G, "graph_ms": 1e3 * t_graph, "plain_ms": 1e3 * t_plain,
            "per_subbox_loop_ms": 1e3 * t_loop, "graph_samples_per_s": G / t_graph,
            "plain_samples_per_s": G / t_plain, "loop_samples_per_s": G / t_loop,
            "launch_variants": {"locate": variants[0], "eval": variants[1]},
            "vertices": plan.n_verts, "tetrahedra": plan.n_tets,
            "vertices_per_subbox": {"min": min(counts), "median": int(np.median(counts)), "max": max(counts)},
            "walk": {k: st[k] for k in ("n_samples_located", "n_walk_steps", "n_exact_tests", "n_ties", "n_outside")},
            "host_plan_s": t_plan,
            "note": "loop timed by wall clock around 64 synchronous C ABI call pairs (what one launch sequence "
                    "per sub-box costs); graph and plain by CUDA events on the handle's stream"}


def sampling_leg(args, local: int, threads: int, cpu: bool) -> dict:
    """Redshift-cone bins and user sampling points (interpolateRedshiftCone,
    interpolateUserSampling).  DTFE() runs both on one tessellation of the
    whole padded box (no sub-box split, src/DTFE.cpp:301), so this leg builds
    a single-box plan: n^3 Zel'dovich particles (n = --sampling-n, rms 1.0
    spacing, velocities as the main workload, periodic 100 Mpc/h, padding 5).
    Cone: apex at the box centre, r in [1, 86.6] (the box corner), theta
    [0, 180], psi [0, 359], n^3 bins.  Points: n^3 uniform points in the box.
    Density, velocity and velocity gradient.  GPU: the cone into device
    outputs (dtfe_gpu_interpolate_cone_dev) and, end to end with host
    buffers, the cone and the points (dtfe_gpu_interpolate_cone /
    _points); CUDA events on the handle's stream.  Reference: the harness's
    interpolateRedshiftCone on every 8th r bin's worth (n/8 bins over the same
    r range) and interpolateUserSampling on the first n^3/8 points, one host
    thread as DTFE() runs them, given the GPU's vertex densities; the GPU
    runs the same reduced cone and points and must match them bit for bit."""
    import torch
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    from dtfe_b200.device import DeviceDTFE
    n = args.sampling_n
    fields = ["density", "velocity", "velocity_gradient"]
    pos, psi = S.zeldovich_lattice(n, S.BOX, 1.0, seed=21)
    rng = np.random.default_rng(22)
    vel = (100.0 * psi / (S.BOX / n) + rng.normal(0.0, 50.0, psi.shape)).astype(np.float32)
    del psi
    w = np.ones(len(pos), np.float32)
    t0 = time.time()
    plan = P.make_plan(pos, w, vel, None, grid=(n, n, n), n_threads=1,
                       average_density_value=float(len(pos)) / S.BOX ** 3)
    t_plan = time.time() - t0
    half = S.BOX / 2
    cone = (1.0, float(np.sqrt(3.0) * half), 0.0, 180.0, 0.0, 359.0)
    origin = (half, half, half)
    dims = (n, n, n)
    G = n ** 3
    pts = rng.uniform(0.0, S.BOX, (G, 3)).astype(np.float32)
    region = [0.0, S.BOX, 0.0, S.BOX, 0.0, S.BOX]
    cuda = f"cuda:{local}"
    outs = {f: torch.empty((G, [1, 3, 9][i]), dtype=torch.float32, device=cuda) for i, f in enumerate(fields)}
    res = {"workload": f"zeldovich{n} single box: {n}^3 particles, {plan.n_verts} vertices, {plan.n_tets} "
                       f"tetrahedra; cone r [1, 86.6] theta [0, 180] psi [0, 359] from the box centre, "
                       f"{n}^3 bins; {G} uniform user points",
           "fields": fields, "plan_s": t_plan}
    with DeviceDTFE(local, 0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        stream = torch.cuda.ExternalStream(dev.stream, device=cuda)

        # padded-box selection with the 27 periodic images (findParticlesInBox)
        # of the n^3 particles: device vs the host restatement on all threads
        pad = 5.0 * S.BOX / n
        full = [0.0, S.BOX, 0.0, S.BOX, 0.0, S.BOX]
        padded = [-pad, S.BOX + pad, -pad, S.BOX + pad, -pad, S.BOX + pad]
        pos_dev = torch.from_numpy(pos).to(cuda)
        for _ in range(2):
            dev.select_in_box(pos_dev, full, padded)
        torch.cuda.synchronize()
        t0 = time.time()
        sel_i, sel_p = dev.select_in_box(pos_dev, full, padded)
        torch.cuda.synchronize()
        t_sel = time.time() - t0
        t0 = time.time()
        h_i, h_p = P.select_in_box(pos, full, padded, True)
        t_host = time.time() - t0
        res["selection"] = {"particles": G, "selected": int(sel_i.numel()), "gpu_ms": 1e3 * t_sel,
                            "host_ms": 1e3 * t_host,
                            "bit_exact_vs_host": bool(np.array_equal(sel_i.cpu().numpy(), h_i) and
                                                      np.array_equal(sel_p.cpu().numpy(), h_p)),
                            "timing": "wall clock around the call (count, scan, one host sync, write)"}
        del pos_dev, sel_i, sel_p

        def timed(fn, k=5):
            for _ in range(2):
                fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                fn()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / 1e3 / k

        t_dev = timed(lambda: dev.interpolate_cone_dev(fields, cone, origin, dims, outs))
        t_cone = timed(lambda: dev.interpolate_cone(fields, cone, origin, dims), 3)
        t_pts = timed(lambda: dev.interpolate_points(fields, pts, region), 3)
        res["cone"] = {"samples_per_s": G / t_dev, "ms": 1e3 * t_dev, "gpu_launches_per_call": 2,
                       "e2e_samples_per_s": G / t_cone, "e2e_ms": 1e3 * t_cone,
                       "d2h_bytes": 4 * 13 * G}
        res["points"] = {"e2e_points_per_s": G / t_pts, "e2e_ms": 1e3 * t_pts, "h2d_bytes": 12 * G,
                         "d2h_bytes": 4 * 13 * G}
        if cpu:
            try:
                import refharness as R
                have = R.available()
            except ImportError:
                have = False
            if have:
                dens = dev.download_vertex_density(plan.n_verts)
                rdims = (max(1, n // 8), n, n)
                ref_c, sec_c = R.run_cone(plan, cone, origin, rdims, dens, timing=True)
                m = G // 8
                ref_p, sec_p = R.run_points(plan, pts[:m], region, dens, timing=True)
                got_c = dev.interpolate_cone(fields, cone, origin, rdims)
                got_p = dev.interpolate_points(fields, pts[:m], region)
                same = all(np.array_equal(got_c[f].reshape(ref_c[f].shape), ref_c[f]) and
                           np.array_equal(got_p[f].reshape(ref_p[f].shape), ref_p[f]) for f in fields)
                nc = int(np.prod(rdims))
                res["reference"] = {
                    "kind": "reference", "cores": 1,
                    "cone_samples_per_s": nc / sec_c, "points_per_s": m / sec_p,
                    "sample": f"cone with {rdims[0]} r bins over the same range ({nc} bins), the first {m} "
                              "points; the reference's own functions on one host thread",
                    "bit_exact_vs_gpu": bool(same)}
    return res


def output_leg(dev, outs: dict, cpu: bool) -> dict:
    """Binary output files (outputFileType 101): the step's device fields
    written as writeOutputData names them, streamed from HBM through pinned
    buffers (dtfe_gpu_write_binary_dev), into a temporary directory; beside
    it the reference's own writeOutputData (harness) writing the same fields
    from host Quantities.  Wall-clock seconds around the whole write (file
    I/O is the bound); the files are compared byte for byte and removed."""
    import shutil
    import tempfile
    import torch
    from dtfe_b200 import output as OUT
    d = tempfile.mkdtemp(prefix="dtfe_out_")
    try:
        torch.cuda.synchronize()
        nbytes = sum(t.numel() * 4 for t in outs.values())
        t0 = time.time()
        mine = OUT.write_fields(os.path.join(d, "gpu"), outs, device=dev)
        t_gpu = time.time() - t0
        res = {"fields": list(outs), "bytes": nbytes, "gpu_s": t_gpu, "gpu_gbs": nbytes / t_gpu / 1e9,
               "files": [os.path.basename(p) for p in mine], "timing": "wall clock (file I/O)"}
        if cpu:
            try:
                import refharness as R
                have = R.available()
            except ImportError:
                have = False
            if have:
                host = {f: t.cpu().numpy() for f, t in outs.items()}
                n = next(iter(host.values())).shape[0]
                t0 = time.time()
                R.write_output(os.path.join(d, "ref"), n, host, {})
                t_ref = time.time() - t0
                same = True
                for p in mine:
                    q = os.path.join(d, os.path.basename(p).replace("gpu", "ref", 1))
                    with open(p, "rb") as f1, open(q, "rb") as f2:
                        while same:
                            a, b = f1.read(1 << 24), f2.read(1 << 24)
                            same = a == b
                            if not a:
                                break
                res["reference"] = {"s": t_ref, "gbs": nbytes / t_ref / 1e9, "kind": "reference", "cores": 1,
                                    "sample": "the same fields from host vectors (writeOutputData, binary)",
                                    "bytes_identical": bool(same)}
        return res
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = host_threads(args.threads)
    plan = build_workload(args.n, 0, threads)
    G = int(np.prod(plan.grid))
    times = []
    import refharness as R
    if R.available():
        kind, cores = "reference", min(threads, plan.n_boxes)
        sample = (f"per step the whole workload: the reference's own vertexDensity + interpolateGrid (density, "
                  f"velocity, velocity gradient; compiled from its sources with its Makefile's -frounding-math "
                  f"-O3) on all {plan.n_boxes} sub-boxes, one host thread each as its DTFE_parallel, then its "
                  f"computeDivergenceShearVorticity on the main grid; step = slowest thread + derived pass")
        for it in range(args.warmup + args.steps):
            t, _ = reference_code_step(plan, threads)
            if it >= args.warmup:
                times.append(t)
    else:
        import copy
        import oracle as O
        from dtfe_b200 import _native as N
        kind, cores = "port", threads
        b0 = plan.boxes[0]
        sub = copy.copy(plan)
        boxes = (N.Subbox * 1)()
        boxes[0] = b0
        sub.boxes = boxes
        per_slab = int(b0.tile_dims[1]) * int(b0.tile_dims[2])
        slabs = max(1, min(int(b0.tile_dims[0]), 2))
        boxes[0].tile_dims[0] = slabs
        cells = slabs * per_slab
        sample = (f"per step: vertex densities of all {plan.n_verts} vertices + {cells} of {G} cells, scaled to "
                  f"the full grid (oracle port)")
        for it in range(args.warmup + args.steps):
            t0 = time.time()
            d32, d64, _ = O.vertex_density(plan)
            t1 = time.time()
            O.interpolate(sub, d32, d64, FIELDS, mode=O.MODE_REF, nthreads=threads)
            t2 = time.time()
            if it >= args.warmup:
                times.append((t1 - t0) + (t2 - t1) * G / cells)
    t_step = float(np.mean(times))
    value = G / t_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "grid samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args, plan, 1),
        "cpu_baseline": {"value": value, "unit": "grid samples/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "grid samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_split(args):
    """One n^3 box split over the ranks: the reference's decomposition into
    ranks x parts sub-boxes (DTFE_parallel's split, src/DTFE.cpp:287-385),
    the sub-boxes dealt to ranks by particle count (dtfe_b200/shard.py), each
    rank tessellating and interpolating only its own; every step ends with
    the tiles gathered to rank 0 through device memory (packed by a kernel,
    NCCL gather, unpacked by a kernel: copySubgridResultsToMain,
    src/subpartition.h:399-432).  Total work is fixed: strong scaling."""
    import datetime
    import torch
    import torch.distributed as dist
    from dtfe_b200 import _native as NF
    from dtfe_b200 import shard as SH
    from dtfe_b200 import synthetic as S
    from dtfe_b200.device import DeviceDTFE
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n = args.n
    threads = max(1, host_threads(args.threads) // world)
    parts = max(1, 16 // world)
    t0 = time.time()
    pos, psi = S.zeldovich_lattice(n, S.BOX, 1.0, seed=1)
    vel = (100.0 * psi / (S.BOX / n) + np.random.default_rng(2).normal(0.0, 50.0, psi.shape)).astype(np.float32)
    del psi
    w = np.ones(len(pos), np.float32)
    plan, mine = SH.make_rank_plan(pos, w, vel, None, grid=(n, n, n), world=world, rank=rank, parts_per_rank=parts,
                                   average_density_value=float(len(pos)) / S.BOX ** 3)
    t_plan = time.time() - t0
    del pos, vel
    G = n ** 3
    fields = FIELDS
    ncomp = {f: NF.field_components(NF.FIELD_SLOTS[f], 0) for f in fields}
    dev = DeviceDTFE(local, 0)
    dev.load(plan)
    outs = {f: torch.zeros((G, ncomp[f]), dtype=torch.float32, device=f"cuda:{local}") for f in fields}
    stream = torch.cuda.ExternalStream(dev.stream, device=f"cuda:{local}")
    tables = SH._exchange_tables(plan, None, f"cuda:{local}") if world > 1 else None

    def step():
        dev.vertex_density(plan.rho_bar)
        dev.interpolate_dev_async(fields, outs, method=0)
        if world > 1:
            dev.synchronize()
            SH.gather_fields_dev(dev, plan, outs, root=0, tables=tables)

    for _ in range(args.warmup):
        step()
    dev.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = dev.read_status()
    t_total = ev0.elapsed_time(ev1) / 1e3
    if world > 1:
        t = torch.tensor([t_total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_total = float(t.item())
    line = {
        "metric": METRIC, "value": G * args.steps / t_total, "unit": "grid samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"zeldovich{n} split over {world} ranks: {n}^3 Zel'dovich particles (rms 1.0 spacing, "
                               f"periodic 100 Mpc/h, padding 5) -> {n}^3 grid, cell-centre "
                               "density+velocity+gradient+div/shear/vort, vertex densities included, tiles gathered "
                               "to rank 0 every step",
                   "subboxes": world * parts, "subboxes_this_rank": len(mine), "vertices_this_rank": plan.n_verts,
                   "l2": "inputs larger than L2 (tessellation arrays > 126 MB)",
                   "parallelism": f"split{world} (sub-boxes dealt to ranks, NCCL tile gather)"},
        "gpu_launches": None, "clocks": clk, "e2e": None, "roofline": None, "cpu_baseline": None,
        "walk": {k: st[k] for k in ("n_samples_located", "n_walk_steps", "n_outside")},
        "host_prep_s": {"plan_s": t_plan},
    }
    dev.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    from dtfe_b200.device import DeviceDTFE

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    threads = max(1, host_threads(args.threads) // max(1, world if world > 1 else 1))
    plan = build_workload(args.n, rank, threads, args.scalars)
    G = int(np.prod(plan.grid))
    from dtfe_b200 import _native as NF
    # the step's fields: the six velocity-derived ones, plus the scalars and
    # their gradients when the workload carries scalars
    fields = FIELDS + (["scalar", "scalar_gradient"] if args.scalars else [])
    ncomp = {f: NF.field_components(NF.FIELD_SLOTS[f], args.scalars) for f in fields}

    dev = DeviceDTFE(local, args.scalars)
    dev.load(plan)
    outs = {f: torch.empty((G, ncomp[f]), dtype=torch.float32, device=f"cuda:{local}") for f in fields}
    stream = torch.cuda.ExternalStream(dev.stream, device=f"cuda:{local}")

    def step():
        dev.vertex_density(plan.rho_bar)
        return dev.interpolate_dev(fields, outs, method=0)

    dev.vertex_density(plan.rho_bar)
    if args.variants:
        variants = tuple(int(x) for x in args.variants.split(","))
        dev.set_variants(*variants)
    else:
        variants = dev.autotune(fields)

    for _ in range(args.warmup):
        step()
    dev.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ki0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ki1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    ev0.record(stream)
    status = None
    # steps queued back to back (dtfe_gpu_interpolate_dev_async); the walk
    # counters are read once the timed region has ended
    for i in range(args.steps):
        dev.vertex_density(plan.rho_bar)
        ki0[i].record(stream)
        dev.interpolate_dev_async(fields, outs, method=0)
        ki1[i].record(stream)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    status = dev.read_status()
    clk = clocks.stop()
    t_total = ev0.elapsed_time(ev1) / 1e3
    t_interp = float(np.mean([a.elapsed_time(b) for a, b in zip(ki0, ki1)])) / 1e3
    if world > 1:
        t = torch.tensor([t_total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_total = float(t.item())
        dist.barrier()
    value = world * G * args.steps / t_total
    ms_step = 1e3 * t_total / args.steps

    # Monte-Carlo average (8 points per cell): point evaluations/s
    # the side legs (MC, comparison estimators, batched sub-boxes, backward)
    # describe one GPU; at N > 1 only the step and its e2e are measured
    side = world == 1
    mc = None
    if side and not args.no_mc:
        for _ in range(2):
            dev.vertex_density(plan.rho_bar)
            dev.interpolate_dev(fields, outs, method=2, n_samples=8, seed=3)
        dev.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            dev.vertex_density(plan.rho_bar)
            dev.interpolate_dev(fields, outs, method=2, n_samples=8, seed=3)
        e1.record(stream)
        e1.synchronize()
        tm = e0.elapsed_time(e1) / 3e3
        mc = {"cells_per_s": G / tm, "point_evals_per_s": 9 * G / tm, "ms_per_step": 1e3 * tm,
              "n_samples": 8, "method": 2}

    # averaging method 1 (the reference's default: 100 points per cell on
    # average, placed in the tetrahedra): grid cells/s of whole steps
    m1 = None
    if side and not args.no_m1:
        from dtfe_b200 import _native as N1
        for _ in range(2):
            dev.vertex_density(plan.rho_bar)
            dev.interpolate_dev(fields, outs, method=N1.METHOD_TETRAHEDRA, n_samples=args.m1_points)
        dev.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            dev.vertex_density(plan.rho_bar)
            dev.interpolate_dev(fields, outs, method=N1.METHOD_TETRAHEDRA, n_samples=args.m1_points)
        e1.record(stream)
        e1.synchronize()
        tm = e0.elapsed_time(e1) / 3e3
        m1 = {"cells_per_s": G / tm, "ms_per_step": 1e3 * tm, "n_points": args.m1_points, "method": 1}
        if rank == 0 and not args.no_cpu:
            m1["reference"] = reference_method1(plan, host_threads(args.threads), args.m1_points)

    # the averaging legs overwrote the step's outputs: one untimed step puts
    # the cell-centre fields back for the output-file leg and the FP64 check
    if side and (mc is not None or m1 is not None):
        step()
        dev.synchronize()

    # end to end through the C ABI with host buffers (pinned)
    e2e = None
    if args.e2e_steps > 0:
        from copy import copy as _copy
        hp = _copy(plan)

        def pin(a):
            if a is None:
                return None
            t = torch.empty(a.shape, dtype={np.dtype("float32"): torch.float32, np.dtype("int32"): torch.int32,
                                            np.dtype("uint8"): torch.uint8}[a.dtype], pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
        from dtfe_b200 import plan as PL
        hp.tet_v, hp.tet_n, hp.xyz = pin(plan.tet_v), pin(plan.tet_n), pin(plan.xyz)
        hp.weight, hp.velocity = pin(plan.weight), pin(plan.velocity)
        # the tessellation as the planner caches it for the transfer: its
        # vertices packed (dtfe_tets_pack_vertices); the device derives the
        # neighbours
        packed = pin(PL.pack_tet_vertices(plan.tet_v))
        # the input particles cross once; each padded vertex is a 4-byte code
        # (source particle, periodic image) that a kernel expands
        codes, box_len = PL.vertex_codes(plan, plan.particles["pos"])
        parts = {"pos": pin(plan.particles["pos"]), "weight": pin(plan.particles["weight"]),
                 "velocity": pin(plan.particles["velocity"]), "scalar": pin(plan.particles["scalar"]),
                 "codes": pin(codes.view(np.int32)).view(np.uint32), "box_length": box_len}
        host_out = {f: pin(np.empty((G, ncomp[f]), np.float32)) for f in fields}
        h_tables = 4 * (len(hp.xs) + len(hp.ys) + len(hp.zs))
        h_vert = hp.xyz.nbytes + hp.weight.nbytes + hp.velocity.nbytes + h_tables
        h_parts = sum(a.nbytes for k, a in parts.items() if k != "box_length" and a is not None) + h_tables
        d2h = sum(a.nbytes for a in host_out.values())

        def e2e_packed():
            dev.upload_packed_particles(hp, packed, parts)
            dev.set_subboxes(hp)
            dev.vertex_density(hp.rho_bar)
            dev.interpolate(fields, method=0, out=host_out)

        def e2e_plain():
            dev.load(hp)
            dev.vertex_density(hp.rho_bar)
            dev.interpolate(fields, method=0, out=host_out)

        def time_e2e(fn):
            fn()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                fn()
            dev.synchronize()
            te = (time.perf_counter() - t0) / args.e2e_steps
            if world > 1:
                t = torch.tensor([te], device=f"cuda:{local}", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                te = float(t.item())
            return te
        te_lat = time_e2e(e2e_packed)
        te_plain = time_e2e(e2e_plain)
        # multiple buffering across steps: a ring of handles, each step's
        # transfers and kernels queued asynchronously, so one handle's
        # downloads and kernels overlap the next one's uploads (every step
        # still moves its inputs in and all its fields out); with three, a
        # step's upload no longer waits for the download two steps back
        nbuf = max(2, args.e2e_buffers)
        ring = [dev]
        for _ in range(nbuf - 1):
            d = DeviceDTFE(local, args.scalars)
            d.set_variants(*variants)
            ring.append(d)
        outs2 = [host_out] + [{f: pin(np.empty_like(a)) for f, a in host_out.items()} for _ in range(nbuf - 1)]
        for d in ring:
            d.upload_packed_particles(hp, packed, parts)
            d.set_subboxes(hp)
        # the handles' inputs cross PCIe one after the other, in step order
        for i, d in enumerate(ring):
            d.chain_uploads(ring[i - 1])

        def e2e_pipelined(k):
            d = ring[k % nbuf]
            d.synchronize()
            d.upload_packed_particles(hp, packed, parts)
            d.vertex_density(hp.rho_bar)
            d.interpolate_async(fields, outs2[k % nbuf], method=0)
        for k in range(nbuf):
            e2e_pipelined(k)
        for d in ring:
            d.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for k in range(args.e2e_steps):
            e2e_pipelined(k)
        for d in ring:
            d.synchronize()
        te = (time.perf_counter() - t0) / args.e2e_steps
        if world > 1:
            t = torch.tensor([te], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        st2 = ring[(args.e2e_steps - 1) % nbuf].read_status()
        for d in ring:
            d.chain_uploads(None)
        for d in ring[1:]:
            d.close()
        e2e = {"value": world * G / te, "unit": "grid samples/s", "h2d_bytes_per_step": int(packed.nbytes + h_parts),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * te,
               "path": "per step: dtfe_gpu_upload_packed_particles (vertex-only packed tetrahedra, neighbours "
                       "derived on the device; the input particles once plus a 4-byte source/image code per "
                       "padded vertex) + vertex_density + interpolate_async into pinned host "
                       f"buffers, {nbuf} handles in turn (uploads chained in step order); sub-box geometry set "
                       "once per handle", "buffers": nbuf,
               "packed_bytes_per_tet": packed.nbytes / plan.n_tets,
               "particles": len(parts["pos"]), "padded_vertices": plan.n_verts,
               "samples_located_last_step": st2["n_samples_located"],
               "single_step_latency_ms": 1e3 * te_lat,
               "unpacked_single_step": {"value": world * G / te_plain, "ms_per_step": 1e3 * te_plain,
                                        "h2d_bytes_per_step": int(hp.tet_v.nbytes + hp.tet_n.nbytes + h_vert)}}

    peak, peak_kind = measured_peak()
    b_alg = 16 * plan.n_tets + plan.n_verts * (12 + 4 + 12 + 4 * args.scalars) + 4 * sum(ncomp.values()) * G
    achieved = b_alg / t_interp / 1e9
    # the interpolation kernel(s) of the chosen locate variant: 9..11 walk and
    # evaluate in one kernel, 3..8 walk then evaluate
    fused = variants[0] >= 9
    traffic = (profile_traffic() or {}).get("fused" if fused else "separate")
    kname = ("k_locate_eval (walk + evaluation in one kernel)" if fused
             else "k_locate_cells + k_eval_centre (cell-centre interpolation)")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                # the ncu capture's DRAM bytes scaled by this launch's algorithmic bytes
                "traffic": (int(traffic["dram_bytes_measured"] * b_alg / traffic["algorithmic_bytes_measured_case"])
                            if traffic else None),
                "kernel": kname, "kernel_ms": 1e3 * t_interp,
                "algorithmic_bytes": int(b_alg), "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})"}

    compare = None
    if side and not args.no_compare:
        compare = compare_leg(args, plan, local, threads, rank == 0 and world == 1 and not args.no_cpu)

    batch = None
    if side and not args.no_batch:
        batch = batch_leg(args, local, threads)

    bwd = None
    if side and not args.no_bwd:
        bwd = backward_leg(args, local, threads)

    output = None
    if side and not args.no_output:
        output = output_leg(dev, {f: outs[f] for f in ("density", "velocity", "velocity_gradient")},
                            rank == 0 and not args.no_cpu)

    sampling = None
    if side and not args.no_sampling:
        sampling = sampling_leg(args, local, threads, rank == 0 and not args.no_cpu)

    tess = None
    if side and not args.no_tess:
        tess = tessellation_leg(plan)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        check = (outs, fields, args.fp64_cells) if args.fp64_cells > 0 else None
        cpu = cpu_baseline(plan, host_threads(args.threads), args.cpu_seconds, args.cpu_kind, check)

    line = {
        "metric": METRIC, "value": value, "unit": "grid samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, plan, world),
        # per step: volumes + seeds, vertex densities, the walk and evaluation
        # (one fused kernel or two), the outside-pencil pass
        "gpu_launches": (4 if variants[0] >= 9 else 5) * args.steps,
        "launch_variants": {"locate": variants[0], "eval": variants[1]},
        "clocks": clk,
        "e2e": e2e,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "mc": mc, "method1": m1,
        "backward": bwd,
        "batched_subboxes": batch,
        "sampling": sampling,
        "output_files": output,
        "comparison_estimators": compare,
        "walk": {k: status[k] for k in ("n_samples_located", "n_walk_steps", "n_exact_tests", "n_ties",
                                        "n_outside")} if status else None,
        # error of the step's fields against the FP64 oracle on sampled cells
        "fp64_error": ({"cells": cpu["fp64_check"]["cells"],
                        "rms_floor": {f: float("%.3g" % v) for f, v in
                                      cpu["fp64_check"]["max_rel_err_rms_floor"].items()},
                        "plain_above_1pct_rms": {f: float("%.3g" % v) for f, v in
                                                 cpu["fp64_check"]["max_rel_err_plain_above_1pct_rms"].items()},
                        "bar": 1e-5}
                       if cpu and cpu.get("fp64_check") else None),
        "host_prep_s": plan.timings,
        "tessellation": tess,
    }
    dev.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.split:
        return run_split(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
