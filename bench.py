#!/usr/bin/env python
"""DOF-stage updates/s of the DG residual + SSP-RK3 time step on B200.

Workload: synthetic NACA 0012 O-grid, 256 x 128 quads -> 65,536 triangles, p = 2 Dubiner basis
(6 modes, 6-point triangle / 3-point edge rules), Euler gamma = 1.4, M = 0.8, AoA = 1.25 deg,
uniform free-stream start, HLLC + slip wall + characteristic far field, KXRCF/WENO limiter after
every stage, SSP-RK3 with CFL 0.1 -- the transonic limiter configuration, computed in FP64.

One step = one iteration of the reference's time_march loop (CFL time step + three RK stages,
each residual + stage update + limiter).  DOF = elements * 4 variables * 6 modes; a step
updates 3 * DOF DOF-stages.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank advances its own replica of the workload (the path does not
shard: replicas only); the timed region is bracketed by barriers and the slowest rank's time
is reported.  ``--impl reference`` times the reference's CPU algorithm (the C++ restatement in
oracle/, since the Rust reference cannot be built here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NI, NJ, ORDER = 256, 128, 2
MACH, AOA, CFL, HCR = 0.8, 1.25, 0.1, 1.4
RHO_INF, P_INF = 1.0, 1.0 / 1.4
WORKLOAD = ("naca0012_ogrid_256x128_p2: 65,536 triangles, 6 modes, M=0.8, AoA=1.25deg, "
            "HLLC, WENO/KXRCF limiter on, SSP-RK3 CFL=0.1, FP64")
METRIC = "DOF-stage updates/s"
# the workload as both arms report it (identical dicts: the reference arm and the GPU arm)
CONFIG = {"workload": WORKLOAD, "elements": 2 * NI * NJ, "order": ORDER, "dof_stage_per_step": 3 * 2 * NI * NJ * 4 * 6,
          "l2": "GPU arm: flushed (256 MiB write) before every timed step, per-step CUDA events; "
                "reference arm: host caches as they are",
          "parallelism": "one device per rank (replicas); the reference arm: host threads of rank 0"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the many-instance measurement")
    ap.add_argument("--batched-instances", type=int, default=256)
    ap.add_argument("--batched-steps", type=int, default=1000)
    ap.add_argument("--no-serving", action="store_true", help="skip the request-stream measurement")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP32-vs-FP64 p=3 measurement")
    ap.add_argument("--precision-steps", type=int, default=500)
    ap.add_argument("--precision-c2-steps", type=int, default=2000)
    ap.add_argument("--no-viscous", action="store_true", help="skip the Navier-Stokes residual measurement")
    ap.add_argument("--viscous-steps", type=int, default=200)
    ap.add_argument("--only", choices=["batched", "precision", "serving", "viscous"],
                    help="run one secondary measurement alone and print its JSON (for profiling)")
    ap.add_argument("--serving-requests", type=int, default=48)
    ap.add_argument("--serving-rates", default="20",
                    help="Poisson arrival rates to serve, requests/s, comma-separated (the same seeded requests at "
                         "each rate); e.g. 1,10,50,200 for the sweep")
    ap.add_argument("--serving-max-steps", type=int, default=5000)
    ap.add_argument("--serving-budget-gib", type=float, default=16.0)
    ap.add_argument("--serving-max-active", type=int, default=2 << 20,
                    help="elements of running requests above which new requests wait (work-in-flight cap)")
    ap.add_argument("--profile-case", choices=["c2", "c3", "batch", "batch_per_order"],
                    help="run a fixed launch sequence for ncu (no timing, no autotuning): c2 = the workload "
                         "above, c3 = the 1024 x 512 p = 3 O-grid (M 0.7, AoA 2 deg), batch / batch_per_order = "
                         "the 256-instance batch as one mixed context / one context per order")
    ap.add_argument("--profile-viscous", action="store_true",
                    help="profile case with the Navier-Stokes residual (Prandtl 0.72, gas constant 287)")
    ap.add_argument("--precision", choices=["fp64", "fp32", "fp32_compute", "tf32", "tf32x3"], default="fp64")
    ap.add_argument("--launch", default="128,2368,128,1,0",
                    help="edge threads, edge blocks, element threads, staged limiter detector, edge pass form "
                         "(0 point, 1 lane pair, 2 staged, 3 point at 64 registers), queue limiter schedule "
                         "(profile case; the last two may be left out: 0)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_mesh():
    from dgm_in_rust_b200 import freestream_quantity, naca0012_ogrid, process_mesh
    raw = naca0012_ogrid(NI, NJ)
    mesh = process_mesh(raw, freestream_quantity(MACH, AOA, RHO_INF, P_INF, HCR), HCR)
    return raw, mesh


def dofs_per_step(ne, nb):
    return ne * 4 * nb * 3


# ------------------------------------------------------------------------------------------
# CPU (reference algorithm) timing
# ------------------------------------------------------------------------------------------
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def time_cpu(raw, steps, warmup, threads, budget_s=None):
    """Time the oracle's time_march on the full workload; returns (DOF-stage/s, steps timed)."""
    from oracle.oracle import Oracle
    o = Oracle(raw=raw, order=ORDER, ncell_gp=6, nedge_gp=3, hcr=HCR, cfl=CFL, final_time=1.0e30,
               final_step=10 ** 9, limiter=True, threads=threads, freestream=(AOA, MACH, RHO_INF, P_INF))
    U = o.initial_solution()
    R = o.new_state()
    for _ in range(warmup):
        o.rk3(R, U, o.compute_time_step(U))
    done, t0 = 0, time.perf_counter()
    while done < steps:
        o.rk3(R, U, o.compute_time_step(U))
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return dofs_per_step(o.ne, o.nb) * done / el, done, el


def mapped_libraries():
    """Shared libraries of this repository mapped into the process (from /proc/self/maps), as
    paths relative to the repository: evidence of which native code a run used."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(ROOT + os.sep):
                    out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def run_reference(args):
    """The reference's CPU algorithm on the host cores, on the same workload, steps and warm-up as
    the GPU arm.  The mesh is generated by the pure-numpy O-grid generator and processed by the
    oracle itself (process_mesh restated), so this arm maps no library of the product."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from dgm_in_rust_b200.mesh import naca0012_ogrid
    raw = naca0012_ogrid(NI, NJ)
    threads = cpu_threads()
    value, done, el = time_cpu(raw, args.steps, args.warmup, threads, budget_s=240.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": args.gpus,
        "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(CONFIG),
        "execution": f"{threads} host threads",
        "cpu_baseline": {"value": value, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                         "sample": f"{done} full RK3 steps of the workload after {args.warmup} warm-up steps; C++ "
                                   "restatement of the reference CPU algorithm (Rust reference not buildable "
                                   "here), OpenMP over volume/edge/boundary passes, serial limiter and dt"},
        "e2e": {"value": value, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["libraries_loaded"] = mapped_libraries()
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while the timed region runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle",
               0x2: "applications_clocks_setting"}

    def __init__(self, device_index):
        self.samples, self.reasons_seen, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            try:
                self._h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
            except Exception:
                self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons_seen.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons_seen), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons_seen), "samples": len(self.samples)}


# phase 3, the limiter, is two launches: the KXRCF detection and the cooperative wave kernel
PHASES = {0: "k_time_step", 1: "k_edge_flux", 2: "k_element", 3: "k_lim_detect+k_limiter"}


def phase_bytes(phase, mesh, nb, n_int, n_bnd):
    """Algorithmic DRAM bytes of one launch of each kernel (FP64): state arrays counted once,
    geometry/connectivity at their stored width, edge-flux intermediates once."""
    ne = mesh.n_elements
    s = 8
    state = ne * 4 * nb * s
    ng = 3
    flux = (n_int + n_bnd) * ng * 4 * s
    if phase == 0:
        return state + ne * 8
    if phase == 1:
        return state + n_int * (8 + 4 + 32) + n_bnd * (4 + 4 + 32) + flux
    if phase == 2:
        return 3 * state + ne * (8 + 32 + 12) + flux
    # limiter: KXRCF reads the state once (neighbour traces come from the same array), face and
    # neighbour ids, h^1.5, per-edge normal/length; writes flags and status words
    return state + ne * (12 + 12 + 8 + 1 + 4) + n_int * 32


def load_traffic():
    """Per-element DRAM traffic of each kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic_c2.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) == 3 and parts[0].startswith("k_"):
                try:
                    out[parts[0]] = (float(parts[1]), float(parts[2]))  # bytes per launch, elements
                except ValueError:
                    pass
    return out


# ------------------------------------------------------------------------------------------
# Batched workload: many uneven instances per launch, FP32 vs FP64, vs one at a time
# ------------------------------------------------------------------------------------------
def run_batched(args, local):
    """256 seeded instances (Ni uniform on {32..256}, Nj = Ni/2, Mach U[0.3,0.85], AoA U[-4,6] deg,
    p in {1,2}): DOF-stage updates/s of (a) the FP32 mixed batch -- one context, one stream, every
    kernel of a step one launch over all 256 instances of both orders -- (b) the FP64 mixed batch,
    (c) for comparison, FP32 with one context per order on two streams (autotuned), and (d) FP64
    one instance at a time on a DOF-weighted sample of 32 instances; accuracy of (a) against (b)
    per instance, beside the FP64 conditioning floor (b started from a 1e-13 perturbed state).
    Inputs exceed the L2 (no flush needed); device time by CUDA events."""
    import torch
    from dgm_in_rust_b200 import Batch, build_solver, forces_to_coefficients
    from dgm_in_rust_b200.workloads import batch_instances, instance_mesh
    seed = 2024
    insts = batch_instances(args.batched_instances, seed=seed)
    t_setup = time.perf_counter()
    built = [(inst, *instance_mesh(inst)) for inst in insts]
    groups = {p: [b for b in built if b[0].order == p] for p in (1, 2)}
    index = {id(m): k for k, (_, m, _) in enumerate(built)}  # instance number in the seeded list
    K, W, W2 = args.batched_steps, 3, 2
    res = {"workload": f"{len(insts)} NACA 0012 O-grids, Ni uniform on {{32,...,256}}, Nj = Ni/2, "
                       f"Mach U[0.3,0.85], AoA U[-4,6] deg, p in {{1,2}} (numpy default_rng({seed})), "
                       f"limiter on, CFL 0.1",
           "instances": len(insts), "elements": int(sum(i.elements for i in insts)),
           "dof": int(sum(i.dofs for i in insts)), "steps": K, "warmup": W + W2}

    def batched(precision, perturb=False, mixed=True):
        batches = []
        sets = [(0, built)] if mixed else [(p, items) for p, items in groups.items() if items]
        for p, items in sets:
            b = Batch([m for _, m, _ in items], [inst.order for inst, _, _ in items] if mixed else p, HCR,
                      [CFL] * len(items), [1.0e30] * len(items), [10 ** 12] * len(items), limiter=True, device=local,
                      precision=precision)
            for i, (_, m, init) in enumerate(items):
                b.set_initial(i, init)
                if perturb:  # the FP64 conditioning floor: a start perturbed by 1e-13 (seeded)
                    U0 = b.download(i)
                    U0 *= 1.0 + 1e-13 * np.random.default_rng(100 + i + 1000 * p).standard_normal(U0.shape)
                    b.upload(i, U0)
            batches.append(b)
        for b in batches:
            b.advance(W)
        for b in batches:
            b.synchronize()
        # tune on a developed state (the free-stream start has no troubled cells), then re-warm
        # the step graphs, which tuning resets
        for b in batches:
            b.autotune(repeats=5)
            b.advance(W2)
        for b in batches:
            b.synchronize()
        streams = [torch.cuda.ExternalStream(b._lib.dgm_stream(b.ctx)) for b in batches]
        start = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in batches]
        start.record(streams[0])
        for st in streams[1:]:
            st.wait_event(start)
        for b in batches:
            b.advance(K)
        for st, ev in zip(streams, ends):
            ev.record(st)
        for b in batches:
            st_code = b.synchronize()
            if st_code != 0:
                raise SystemExit(f"batched run failed with status {st_code}")
        ms = max(start.elapsed_time(ev) for ev in ends)
        dev_bytes = sum(int(b._lib.dgm_device_bytes(b.ctx)) for b in batches)
        # end states for the accuracy comparison: C_L / C_D of every instance, the density field
        # of every 8th instance of each group
        acc = {}
        for (p, items), b in zip(sets, batches):
            d = b.diagnostics()
            for i, (inst, m, _) in enumerate(items):
                cl, cd = forces_to_coefficients(d[i, 4], d[i, 5], inst.aoa, 1.0, inst.mach)
                rho = b.download(i)[:, 0].copy() if i % 8 == 0 else None
                mass = b.tables[inst.order][1].mass_mat_diag
                w = (mass[None, :] * (0.5 * m.elem_jacob_det)[:, None]) if rho is not None else None
                acc[(inst.order, index[id(m)])] = (cl, cd, rho, w)
        for b in batches:
            b.close()
        return res["dof"] * 3 * K / (ms * 1e-3), ms / K, dev_bytes, acc

    v32, ms32, bytes32, acc32 = batched("fp32")
    v32c, ms32c, bytes32c, acc32c = batched("fp32_compute")
    v32s, ms32s, _, _ = batched("fp32", mixed=False)
    v64, ms64, bytes64, acc64 = batched("fp64")
    _, _, _, accp = batched("fp64", perturb=True)
    floor_cl = {k: abs(accp[k][0] - acc64[k][0]) for k in acc64}
    floor_cd = {k: abs(accp[k][1] - acc64[k][1]) for k in acc64}

    def versus(acc, tol=1e-4):
        dcl = {k: abs(acc[k][0] - acc64[k][0]) for k in acc64}
        dcd = {k: abs(acc[k][1] - acc64[k][1]) for k in acc64}
        errs = [field_rel_l2(acc[k][2], acc64[k][2], acc64[k][3]) for k in acc64 if acc64[k][2] is not None]
        ok = {k: dcl[k] <= tol and dcd[k] <= tol for k in acc64}
        good = [k for k in acc64 if floor_cl[k] <= tol and floor_cd[k] <= tol]
        return {"steps": W + W2 + K, "max_abs_delta_cl": max(dcl.values()), "max_abs_delta_cd": max(dcd.values()),
                "median_abs_delta_cl": float(np.median(list(dcl.values()))),
                "instances_meeting_1e-4": int(sum(ok.values())),
                "instances_with_fp64_floor_below_1e-4": len(good),
                "of_those_meeting_1e-4": int(sum(ok[k] for k in good)),
                "max_abs_delta_cl_where_floor_below_1e-4": max([dcl[k] for k in good], default=None),
                "density_rel_l2_max": max(errs), "density_rel_l2_median": float(np.median(errs)),
                "density_sample": f"{len(errs)} instances (every 8th of each order group)"}

    res["fp64_conditioning_floor"] = {
        "perturbation": "each instance's initial state x (1 + 1e-13 N(0,1)), FP64, same steps",
        "max_abs_delta_cl": max(floor_cl.values()), "median_abs_delta_cl": float(np.median(list(floor_cl.values()))),
        "max_abs_delta_cd": max(floor_cd.values()),
        "instances_below_1e-4": int(sum(floor_cl[k] <= 1e-4 and floor_cd[k] <= 1e-4 for k in floor_cl)),
        "per_instance_abs_delta_cl": {f"instance_{k[1]}_p{k[0]}": v for k, v in sorted(floor_cl.items(),
                                                                                     key=lambda kv: kv[0][1])}}
    res["fp32_vs_fp64_after_steps"] = versus(acc32)
    res["fp32_compute_vs_fp64_after_steps"] = versus(acc32c)
    # one at a time, FP64: a DOF-weighted sample (every 8th instance in DOF order)
    order = sorted(range(len(built)), key=lambda k: built[k][0].dofs)
    sample = [built[k] for k in order[::max(1, len(built) // 32)]]
    tot_ms, tot_dof = 0.0, 0
    for inst, m, init in sample:
        s = build_solver(m, inst.order, HCR, CFL, 1.0e30, 10 ** 12, limiter=True, device=local)
        td = s.temporal_disc
        td.set_initial_on_device(init)
        td.advance(W)
        td.synchronize()
        st = torch.cuda.ExternalStream(s.spatial_disc._lib.dgm_stream(s.spatial_disc.ctx))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        td.advance(K)
        b.record(st)
        td.synchronize()
        tot_ms += a.elapsed_time(b)
        tot_dof += inst.dofs
        s.close()
    v_single = tot_dof * 3 * K / (tot_ms * 1e-3)
    res.update({
        "fp32_batched": v32, "fp32_compute_batched": v32c, "fp64_batched": v64, "fp64_one_at_a_time": v_single,
        "ms_per_step_fp32_compute_batched": ms32c,
        "speedup_fp32_compute_batched_vs_fp64_one_at_a_time": v32c / v_single,
        "speedup_fp32_compute_batched_vs_fp64_batched": v32c / v64,
        "fp32_one_context_per_order_two_streams": v32s, "ms_per_step_fp32_two_streams": ms32s,
        "launch_structure": "mixed batch: one context, one stream, one launch per kernel of the step over all "
                            "instances of both orders (14 launches per step, CUDA graphs of 8 steps)",
        "ms_per_step_fp32_batched": ms32, "ms_per_step_fp64_batched": ms64,
        "device_bytes_fp32": bytes32, "device_bytes_fp64": bytes64,
        "speedup_fp32_batched_vs_fp64_one_at_a_time": v32 / v_single,
        "speedup_fp32_batched_vs_fp64_batched": v32 / v64,
        "one_at_a_time_sample": f"{len(sample)} instances, every {max(1, len(built) // 32)}th by DOF count",
        "setup_s": time.perf_counter() - t_setup,
    })
    return res


# ------------------------------------------------------------------------------------------
# Precision: FP32 vs FP64 on the large p = 3 workload
# ------------------------------------------------------------------------------------------
def field_rel_l2(a, b, w):
    """Relative L2 error of the fields whose modal coefficients are a, b ([element][mode]); w =
    mass_b * J_e / 2, so sum(w * c^2) is the integral of the square (orthogonal basis)."""
    return float(np.sqrt(np.sum(w * (a - b) ** 2) / np.sum(w * b * b)))


def wall_elements(mesh):
    """Elements with an edge on a wall patch: the first cell layer on the body."""
    bnd = np.nonzero(mesh.edge_elements[:, 1] == -1)[0]
    wall = [d for d in bnd if mesh.patch_type[mesh.edge_patch[d]] == 0]
    return np.unique(mesh.edge_elements[wall, 0])


def accuracy_report(U, U64, cl, cd, cl64, cd64, floor, w, wall, tol=1e-4):
    """Errors of one precision mode against FP64 on the same steps: relative L2 of every field
    (area-weighted, and over the coefficients), relative L2 of the density over the first wall
    layer (coefficients), |dC_L|, |dC_D|, and pass/fail against tol, with the FP64 conditioning
    floor (|dC_L|, |dC_D| of FP64 from a 1e-13 perturbed start) beside it."""
    names = ("rho", "rho_u", "rho_v", "rho_E")
    dcl, dcd = abs(cl - cl64), abs(cd - cd64)
    rho_w = float(np.linalg.norm(U[wall, 0] - U64[wall, 0]) / np.linalg.norm(U64[wall, 0]))
    return {"rel_l2": {n: field_rel_l2(U[:, v], U64[:, v], w) for v, n in enumerate(names)},
            "rel_l2_coefficients": {n: float(np.linalg.norm(U[:, v] - U64[:, v]) / np.linalg.norm(U64[:, v]))
                                    for v, n in enumerate(names)},
            "rel_l2_density_first_wall_layer": rho_w,
            "abs_delta_cl": dcl, "abs_delta_cd": dcd,
            "fp64_floor_abs_delta_cl": floor[0], "fp64_floor_abs_delta_cd": floor[1],
            "meets_1e-4": bool(dcl <= tol and dcd <= tol),
            "floor_below_1e-4": bool(floor[0] <= tol and floor[1] <= tol),
            "within_twice_the_floor": bool(dcl <= 2 * floor[0] and dcd <= 2 * floor[1])}


def precision_case(inst, K, modes, local, label):
    """The same K steps from the free stream in FP64, in each precision mode of ``modes``, and in
    FP64 from a start perturbed by 1e-13 (the conditioning floor); each mode's launch
    configuration tuned on a developed state.  Returns per-mode throughput and accuracy against
    FP64."""
    import torch
    from dgm_in_rust_b200 import build_solver, forces_to_coefficients
    from dgm_in_rust_b200.workloads import instance_mesh
    mesh, init = instance_mesh(inst)
    nb = (inst.order + 1) * (inst.order + 2) // 2
    res = {"workload": label, "steps": K}
    out, tuned = {}, {}
    for prec in ("fp64",) + tuple(modes) + ("fp64_perturbed",):
        mode = "fp64" if prec == "fp64_perturbed" else prec
        if mode not in tuned:
            t = build_solver(mesh, inst.order, HCR, CFL, 1.0e30, 10 ** 12, limiter=True, device=local, precision=mode)
            t.temporal_disc.set_initial_on_device(init)
            t.temporal_disc.advance(20)
            t.temporal_disc.synchronize()
            tuned[mode] = t.spatial_disc.autotune(repeats=5)
            t.close()
        s = build_solver(mesh, inst.order, HCR, CFL, 1.0e30, K, limiter=True, device=local, precision=mode)
        td, sd = s.temporal_disc, s.spatial_disc
        cfg = tuned[mode]
        sd.set_launch_config(cfg["edge_threads"], cfg["edge_blocks"], cfg["element_threads"])
        sd.set_edge_form(cfg["edge_form"])
        sd.set_limiter_detector(cfg["limiter_detector"] == "staged")
        sd.set_limiter_schedule(cfg["limiter_schedule"] == "queue")
        sd.set_limiter_grid(cfg["limiter_grid"] == "one_per_sm")
        td.set_initial_on_device(init)
        if prec == "fp64_perturbed":
            U0 = sd.new_state()
            td.download(U0)
            U0 *= 1.0 + 1e-13 * np.random.default_rng(11).standard_normal(U0.shape)
            td.upload(U0)
            del U0
        st = torch.cuda.ExternalStream(sd._lib.dgm_stream(sd.ctx))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        td.advance(K)
        b.record(st)
        td.synchronize()
        ms = a.elapsed_time(b)
        U = sd.new_state()
        td.download(U)
        d = sd.diagnostics()
        cl, cd = forces_to_coefficients(d[4], d[5], inst.aoa, 1.0, inst.mach)
        troubled, _ = sd.limiter_stats()
        out[prec] = (U, cl, cd)
        if prec != "fp64_perturbed":
            res[prec] = {"dof_stage_updates_per_s": inst.dofs * 3 * td.current_step / (ms * 1e-3),
                         "ms_per_step": ms / max(td.current_step, 1), "steps_done": td.current_step,
                         "time": td.current_time, "cl": cl, "cd": cd, "troubled_cells_last_stage": troubled,
                         "launch": {k: cfg[k] for k in ("edge_threads", "edge_blocks", "element_threads", "edge_form",
                                                        "limiter_detector", "limiter_schedule")}}
        w_basis = s.basis.mass_mat_diag
        s.close()
    U64, cl64, cd64 = out["fp64"]
    Up, clp, cdp = out["fp64_perturbed"]
    w = w_basis[None, :] * (0.5 * mesh.elem_jacob_det)[:, None]
    wall = wall_elements(mesh)
    floor = (abs(clp - cl64), abs(cdp - cd64))
    res["fp64_conditioning_floor"] = {"perturbation": "initial state x (1 + 1e-13 N(0,1)), FP64",
                                      "abs_delta_cl": floor[0], "abs_delta_cd": floor[1],
                                      "rel_l2_rho": field_rel_l2(Up[:, 0], U64[:, 0], w),
                                      "rel_l2_density_first_wall_layer": float(
                                          np.linalg.norm(Up[wall, 0] - U64[wall, 0]) / np.linalg.norm(U64[wall, 0]))}
    for prec in modes:
        U, cl, cd = out[prec]
        res[f"{prec}_vs_fp64"] = accuracy_report(U, U64, cl, cd, cl64, cd64, floor, w, wall)
        res[f"speedup_{prec}_vs_fp64"] = res[prec]["dof_stage_updates_per_s"] / res["fp64"]["dof_stage_updates_per_s"]
    res["wall_layer_elements"] = int(len(wall))
    res["elements"] = int(mesh.n_elements)
    res["dof_per_element"] = 4 * nb
    return res


def run_precision(args, local):
    """FP32 and the tensor-core TF32 modes against FP64 on (a) the precision configuration, NACA
    0012 O-grid 1024 x 512 (1,048,576 triangles), p = 3, M = 0.7, AoA = 2 deg, free-stream start,
    limiter on, CFL 0.1, --precision-steps steps, and (b) a grid of the transonic configuration's
    size with a coarser wall layer, 512 x 64 (65,536 triangles, first cell 4e-4 chords instead of
    5e-8), p = 2, M = 0.5, AoA = 2 deg, --precision-c2-steps steps, where the FP64 solution is
    well conditioned (its 1e-13-perturbation floor is small), so that errors of 1e-4 can be told
    apart.  Reports for each: throughput of every mode, relative L2 errors (area-weighted and
    coefficient-level, and over the first wall layer), |dC_L|, |dC_D|, pass/fail against 1e-4 and
    the FP64 floor.  CUDA events on the library stream."""
    from dgm_in_rust_b200.workloads import Instance
    K = args.precision_steps
    c3 = precision_case(Instance(1024, 512, 0.7, 2.0, 3), K, ("fp32", "fp32_compute", "tf32", "tf32x3"), local,
                        f"naca0012_ogrid_1024x512_p3: 1,048,576 triangles, 10 modes, M=0.7, AoA=2deg, limiter on, "
                        f"CFL 0.1, free-stream start, {K} steps")
    K2 = args.precision_c2_steps
    c2 = precision_case(Instance(512, 64, 0.5, 2.0, 2), K2, ("fp32", "fp32_compute", "tf32x3"), local,
                        f"naca0012_ogrid_512x64_p2: 65,536 triangles, 6 modes, M=0.5, AoA=2deg, limiter on, CFL 0.1, "
                        f"free-stream start, {K2} steps (first wall cell 4e-4 chords)")
    c3["well_conditioned_65536"] = c2
    return c3


# ------------------------------------------------------------------------------------------
# Navier-Stokes residual (the reference's disabled viscous terms) on the transonic workload
# ------------------------------------------------------------------------------------------
def run_viscous(args, local):
    """The transonic workload (256 x 128 O-grid, 65,536 triangles, p = 2, M 0.8, AoA 1.25 deg,
    limiter on, FP64, non-dimensional free stream) with the Navier-Stokes (BR2) residual at the
    reference's parameters (Prandtl 0.72, gas constant 287) against the Euler residual: DOF-stage
    updates/s of each over --viscous-steps steps from the free stream (after 3 warm-up steps), CUDA
    events on the library stream, and the state difference the viscous terms make.  The kernels'
    cost does not depend on the viscosity's size; at these parameters T = p / (R rho) = 0.0025 and
    Sutherland's viscosity is ~1e-12, so the difference is round-off sized.  In the reference's
    dimensional free stream (p = 1e5: Reynolds number ~1.4e7 per chord) this grid's 5e-8-chord wall
    cells make the explicit march unstable at the convective CFL number (negative pressure in the
    second step, the oracle alike), so that case is not timed."""
    import torch
    from dgm_in_rust_b200 import build_solver
    from dgm_in_rust_b200.workloads import Instance, instance_mesh
    inst = Instance(NI, NJ, MACH, AOA, ORDER)
    mesh, init = instance_mesh(inst)
    dofs = inst.dofs
    K, W = args.viscous_steps, 3
    out = {"workload": f"naca0012_ogrid_{NI}x{NJ}_p{ORDER}: {mesh.n_elements} triangles, M={MACH}, AoA={AOA}deg, "
                       f"limiter on, CFL {CFL}, FP64, free-stream start, {K} steps after {W}",
           "prandtl_number": 0.72, "gas_constant": 287.0}
    states = {}
    for visc in (False, True):
        s = build_solver(mesh, ORDER, HCR, CFL, 1.0e30, 10 ** 12, limiter=True, device=local)
        sd, td = s.spatial_disc, s.temporal_disc
        if visc:
            sd.set_viscous(True, 0.72, 287.0)
        td.set_initial_on_device(init)
        td.advance(W)
        td.synchronize()
        st = torch.cuda.ExternalStream(sd._lib.dgm_stream(sd.ctx))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        td.advance(K)
        b.record(st)
        td.synchronize()
        ms = a.elapsed_time(b)
        U = sd.new_state()
        td.download(U)
        states[visc] = U
        key = "navier_stokes" if visc else "euler"
        out[key] = {"dof_stage_updates_per_s": dofs * 3 * K / (ms * 1e-3), "ms_per_step": ms / K,
                    "launches_per_step": int(sd._lib.dgm_launches_per_step(sd.ctx))}
        s.close()
    out["ns_over_euler_time"] = out["navier_stokes"]["ms_per_step"] / out["euler"]["ms_per_step"]
    diff = states[True] - states[False]
    out["state_rel_l2_ns_vs_euler"] = float(np.linalg.norm(diff) / np.linalg.norm(states[False]))
    return out


# ------------------------------------------------------------------------------------------
# Serving: Poisson request stream, continuous batching, vs FP64 one at a time
# ------------------------------------------------------------------------------------------
def run_serving(args, local):
    """A seeded Poisson stream of solve requests (triangles log-uniform in [2e3, 5e5], O-grid
    aspect 2:1, Mach U[0.3,0.85], AoA U[-4,6] deg, p in {1,2,3}), each run to a density-residual
    drop of 1e-6 or the step cap, served (a) by the continuous-batching loop in FP32 with real
    arrival times, an HBM budget and slot reuse, at every rate of --serving-rates, and (b) one
    request at a time on the plain FP64 context, first come first served: service times measured
    back to back once (the requests are the same at every rate: the seed fixes sizes, orders and
    flow conditions, the rate only scales the gaps), latencies from the FIFO queue under each
    rate's arrival times.  Latency = arrival to retirement (time to convergence, or to the step
    cap where the request does not converge); throughput = DOF-stage updates / wall time (a) or /
    total service time (b), host mesh preparation included in both."""
    from dgm_in_rust_b200.serving import ServingLoop, latency_summary, one_at_a_time, requests_from_stream
    from dgm_in_rust_b200.workloads import request_stream
    seed = 7
    rates = [float(x) for x in args.serving_rates.split(",") if x.strip()]
    kw = dict(chunk_steps=32, tol=1e-6, max_steps=args.serving_max_steps)
    budget = int(args.serving_budget_gib * (1 << 30))
    out = {"workload": f"{args.serving_requests} requests per rate, Poisson arrivals (request_stream seed {seed}), "
                       f"triangles log-uniform [2e3, 5e5], p in {{1,2,3}}, Mach U[0.3,0.85], AoA U[-4,6] deg; stop at "
                       f"density-residual drop 1e-6 or {args.serving_max_steps} steps; convergence checked at step 1 "
                       f"then every 32",
           "hbm_budget_bytes": budget, "max_active_elements": args.serving_max_active, "rates": {}}
    base = requests_from_stream(request_stream(args.serving_requests, rates[0], seed=seed))
    out["elements_total"] = int(sum(r.instance.elements for r in base))
    # FP64 one at a time: service times once, FIFO latencies per rate
    alone, busy, prep = one_at_a_time(base, precision="fp64", device=local, **kw)
    service = {r.rid: r.finished_s - r.admitted_s for r in alone}
    gpu_only = sum(r.dofs * 3 * r.steps for r in alone) / max(busy - prep, 1e-9)
    out["fp64_one_at_a_time_service_s"] = busy
    out["fp64_one_at_a_time_excluding_host_prep_dof_stage_per_s"] = gpu_only
    for rate in rates:
        reqs = requests_from_stream(request_stream(args.serving_requests, rate, seed=seed))
        assert [(r.instance.ni, r.instance.order) for r in reqs] == [(r.instance.ni, r.instance.order) for r in base]
        loop = ServingLoop(hbm_budget_bytes=budget, device=local, precision="fp32",
                           max_active_elements=args.serving_max_active, **kw)
        t = time.perf_counter()
        served = loop.run(reqs, realtime=True)
        wall = time.perf_counter() - t
        s32 = latency_summary(served, wall)
        fifo = {r.rid: r for r in alone}
        finish = 0.0
        for r in sorted(reqs, key=lambda q: (q.arrival_s, q.rid)):
            a = fifo[r.rid]
            start = max(r.arrival_s, finish)
            finish = start + service[r.rid]
            a.arrival_s, a.admitted_s, a.finished_s = r.arrival_s, start, finish
        s64 = latency_summary(list(fifo.values()), busy)
        out["rates"][f"{rate:g}"] = {
            "fp32_serving": s32, "fp64_one_at_a_time": s64,
            "peak_resident_bytes": loop.peak_bytes, "cohorts": loop.cohorts_formed, "slot_reuses": loop.slot_reuses,
            "max_concurrent_requests": loop.max_concurrent, "scheduler": loop.stats,
            "throughput_speedup": s32["dof_stage_updates_per_s"] / s64["dof_stage_updates_per_s"],
            "p99_speedup": s64["p99_s"] / s32["p99_s"]}
    return out


def run_ours(args):
    import torch
    world, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from dgm_in_rust_b200 import InitialSolution, build_solver, initial_state
    from dgm_in_rust_b200.build import build
    build()
    raw, mesh = make_mesh()
    solver = build_solver(mesh, ORDER, HCR, CFL, 1.0e30, 10 ** 12, limiter=True, device=local)
    sd, td = solver.spatial_disc, solver.temporal_disc
    L = sd._lib
    ctx = sd.ctx
    U0 = initial_state(mesh, solver.basis, solver.gauss_points, HCR, InitialSolution(RHO_INF, AOA, MACH, P_INF))
    td.upload(U0)
    stream = torch.cuda.ExternalStream(L.dgm_stream(ctx))
    ne, nb = mesh.n_elements, solver.basis.dof
    dps = dofs_per_step(ne, nb)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # W warm-up steps in all: the first max(1, W - 3) develop the state (the free-stream start
    # has no troubled cells) and instantiate the step graphs, the launch configuration is tuned on
    # that state, and the remaining steps rebuild the graphs, which tuning resets
    first = max(1, args.warmup - 3)
    td.advance(first)
    td.synchronize()
    tuned = sd.autotune(repeats=20)
    td.advance(max(args.warmup - first, 0))
    td.synchronize()
    # timed region: K steps, L2 flushed before each step, each step bracketed by events
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    sampler = ClockSampler(local)
    with sampler:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                evs[i][0].record(stream)
            td.advance(1)
            with torch.cuda.stream(stream):
                evs[i][1].record(stream)
        td.synchronize()
    barrier()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    troubled, waves = sd.limiter_stats()
    # L2-resident throughput: the same steps back to back in CUDA graphs (no flush)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with torch.cuda.stream(stream):
        e0.record(stream)
    td.advance(args.steps)
    with torch.cuda.stream(stream):
        e1.record(stream)
    td.synchronize()
    ms_resident = e0.elapsed_time(e1)
    # per-kernel timing (L2 flushed before each launch) for the roofline
    n_int = int(mesh.internal_edge_indices.shape[0])
    n_bnd = int((mesh.edge_elements[:, 1] == -1).sum())
    reps = 20
    kernel_us = {}
    for ph in range(4):
        tot = 0.0
        for r in range(reps + 2):
            if ph == 3:  # the limiter acts on the stage buffer written by phase 2
                L.dgm_launch_phase(ctx, 1)
                L.dgm_launch_phase(ctx, 2)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.fill_(float(r))
                a.record(stream)
            st = L.dgm_launch_phase(ctx, ph)
            if st != 0:
                raise SystemExit(f"dgm_launch_phase({ph}) failed: {st}")
            with torch.cuda.stream(stream):
                b.record(stream)
            td.synchronize()
            if r >= 2:
                tot += a.elapsed_time(b)
        kernel_us[PHASES[ph]] = 1e3 * tot / reps
    share = {k: kernel_us[k] * L.dgm_phase_launches_per_step(ctx, ph) for ph, k in PHASES.items()}
    dom_phase = max(PHASES, key=lambda ph: share[PHASES[ph]])
    dom = PHASES[dom_phase]
    alg = phase_bytes(dom_phase, mesh, nb, n_int, n_bnd)
    peaks = {}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peaks = json.load(f)
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    achieved = alg / (kernel_us[dom] * 1e-6) / 1e9
    tr = load_traffic()
    parts = [tr.get(k) for k in dom.split("+")]
    traffic_per_launch = sum(t[0] * ne / t[1] for t in parts) if all(parts) else None

    # e2e: the reference-facing call per step -- time_march over one iteration with host
    # (pinned) buffers: upload of the state, the step, download of state and residual
    Uh = torch.from_numpy(U0.copy()).pin_memory()
    Rh = torch.zeros_like(Uh).pin_memory()
    Un, Rn = Uh.numpy(), Rh.numpy()
    td.set_clock(0.0, 0)
    for i in range(3):
        td.set_limits(1.0e30, i + 1)
        td.time_march(sd, Rn, Un)
    barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        td.set_limits(1.0e30, 3 + i + 1)
        td.time_march(sd, Rn, Un)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    barrier()
    state_bytes = ne * 4 * nb * 8

    # max over ranks
    vals = torch.tensor([ms, ms_resident, e2e_s], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    ms, ms_resident, e2e_s = [float(v) for v in vals.tolist()]
    value = world * dps * args.steps / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(CONFIG),
        "execution": f"replicas x{world}" if world > 1 else "single GPU",
        "launch": tuned,
        "value_l2_resident": world * dps * args.steps / (ms_resident * 1e-3),
        "e2e": {"value": world * dps * args.steps / e2e_s, "unit": "DOF-stage/s",
                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": 2 * state_bytes,
                "call": "dgm_time_march over one iteration (dgm_set_limits + dgm_time_march), pinned host arrays"},
        "gpu_launches": L.dgm_launches_per_step(ctx) * args.steps,
        "kernel_us": {k: round(v, 3) for k, v in kernel_us.items()},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": alg,
                     "traffic": traffic_per_launch},
        "limiter": {"troubled_cells_last_step": troubled, "waves_last_pass": waves},
        "clocks": sampler.summary(),
    }
    if world == 1 and not args.no_batched:
        line["batched"] = run_batched(args, local)
    if world == 1 and not args.no_precision:
        line["precision"] = run_precision(args, local)
    if world == 1 and not args.no_serving:
        line["serving"] = run_serving(args, local)
    if world == 1 and not args.no_viscous:
        line["viscous"] = run_viscous(args, local)
    # the metric's comparison and latencies, lifted from the secondary measurements
    if "batched" in line:
        b = line["batched"]
        line["batched_fp32_vs_plain_fp64"] = {
            "fp32_batched_dof_stage_per_s": b["fp32_batched"], "fp64_one_at_a_time_dof_stage_per_s": b["fp64_one_at_a_time"],
            "ratio": b["speedup_fp32_batched_vs_fp64_one_at_a_time"],
            "ratio_vs_fp64_batched": b["speedup_fp32_batched_vs_fp64_batched"],
            "fp32_compute_batched_dof_stage_per_s": b["fp32_compute_batched"],
            "fp32_compute_ratio": b["speedup_fp32_compute_batched_vs_fp64_one_at_a_time"], "steps": b["steps"]}
    if "serving" in line:
        line["serving_latency_s"] = {
            rate: {"fp32_serving_p50": r["fp32_serving"]["p50_s"], "fp32_serving_p99": r["fp32_serving"]["p99_s"],
                   "fp64_one_at_a_time_p50": r["fp64_one_at_a_time"]["p50_s"],
                   "fp64_one_at_a_time_p99": r["fp64_one_at_a_time"]["p99_s"],
                   "converged": r["fp32_serving"]["converged"]}
            for rate, r in line["serving"]["rates"].items()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        v, done, el = time_cpu(raw, 1000, 1, threads, budget_s=12.0)
        line["cpu_baseline"] = {"value": v, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                                "sample": f"{done} full RK3 steps ({el:.1f} s) of the workload after 1 warm-up "
                                          "step; C++ restatement of the reference CPU algorithm"}
    if rank == 0:
        line["libraries_loaded"] = mapped_libraries()
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_profile_batch(args):
    """The batching configuration's 256 instances for ncu captures, no autotuning: "batch" is the
    mixed batch (one context, one stream, one launch per kernel of the step over both orders),
    "batch_per_order" one batch per order on its own stream; --warmup + --steps steps."""
    from dgm_in_rust_b200 import Batch
    from dgm_in_rust_b200.workloads import batch_instances, instance_mesh
    built = [(inst, *instance_mesh(inst)) for inst in batch_instances(args.batched_instances, seed=2024)]
    if args.profile_case == "batch":
        sets = [([inst.order for inst, _, _ in built], built)]
    else:
        sets = [(p, [b for b in built if b[0].order == p]) for p in (1, 2)]
    batches = []
    for order, items in sets:
        b = Batch([m for _, m, _ in items], order, HCR, [CFL] * len(items), [1.0e30] * len(items),
                  [10 ** 12] * len(items), limiter=True, precision=args.precision)
        for i, (_, _, init) in enumerate(items):
            b.set_initial(i, init)
        batches.append(b)
    for b in batches:
        b.advance(args.warmup + args.steps)
    status = [b.synchronize() for b in batches]
    print(json.dumps({"profile_case": args.profile_case, "precision": args.precision, "instances": len(built),
                      "contexts": len(batches), "status": status}), flush=True)
    for b in batches:
        b.close()
    return 0 if not any(status) else 1


def run_profile_case(args):
    """A deterministic launch sequence for ncu captures: the case's context (one k_weno_gram and
    one k_project_uniform launch), then --warmup + --steps time-march steps with the launch
    configuration given by --launch, no autotuning.  Every step launches k_step_head,
    3 x (k_edge_flux, k_element or k_element_tc, k_limiter) and k_step_end, so a capture of the
    first step after the warm-up skips 3 * warmup launches of a stage kernel."""
    import torch
    from dgm_in_rust_b200 import build_solver
    from dgm_in_rust_b200.build import build
    from dgm_in_rust_b200.workloads import Instance, instance_mesh
    build()
    torch.cuda.set_device(0)
    if args.profile_case in ("batch", "batch_per_order"):
        return run_profile_batch(args)
    inst = {"c2": Instance(NI, NJ, MACH, AOA, ORDER), "c3": Instance(1024, 512, 0.7, 2.0, 3)}[args.profile_case]
    mesh, init = instance_mesh(inst)
    s = build_solver(mesh, inst.order, HCR, CFL, 1.0e30, 10 ** 12, limiter=True, precision=args.precision)
    sd, td = s.spatial_disc, s.temporal_disc
    vals = [int(x) for x in args.launch.split(",")] + [0, 0]
    e_t, e_b, l_t, staged, pair, queue = vals[:6]
    sd.set_launch_config(e_t, e_b, l_t)
    sd.set_limiter_detector(bool(staged))
    sd.set_limiter_schedule(bool(queue))
    sd.set_edge_form(("point", "pair", "staged", "point_r64")[pair])
    if args.profile_viscous:
        sd.set_viscous(True, 0.72, 287.0)
    td.set_initial_on_device(init)
    td.advance(args.warmup + args.steps)
    td.synchronize()
    troubled, _ = sd.limiter_stats()
    print(json.dumps({"profile_case": args.profile_case, "precision": args.precision, "viscous": sd.viscous,
                      "elements": mesh.n_elements,
                      "steps": td.current_step, "launch": sd.launch_config, "troubled_last_step": troubled}), flush=True)
    s.close()
    return 0


def main():
    args = parse()
    if args.profile_case:
        return run_profile_case(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.only:
        import torch
        from dgm_in_rust_b200.build import build
        build()
        torch.cuda.set_device(0)
        fn = {"batched": run_batched, "precision": run_precision, "serving": run_serving,
              "viscous": run_viscous}[args.only]
        print(json.dumps({args.only: fn(args, 0)}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
