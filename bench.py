"""Throughput of the single-block GRMHD RK2 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c3|c2|c4|c5] [--precision fp64|mixed|both]
                    [--recon ppm|mc] [--riemann hll|hllc|hlld] [--no-accuracy]

Workload (default c3): the 3-D Fishbone-Moncrief torus around a Kerr hole,
a = 0.9375, r_in = 6, r_max = 12, gamma = 13/9, beta_min = 100, 4 % seeded
pressure noise, 384 x 192 x 192 zones (14.2 M cells; c2: 192 x 96 x 64),
synthetic initial data, inputs (~1 GB of primitives) larger than L2.

A step is one RK2 step (half + full sub-step with ghost fills) of every zone.
value = zones x steps / device time (cell-updates/s, the ZCPS of main.c:225),
timed with CUDA events on the stream the kernels run on, after W warm-up
steps, max over ranks. N > 1 runs independent replicas (one block per GPU,
no exchange): scaling "weak".

The default line also carries, untimed: `adjoint` -- the adjoint workload
(2-D torus 256 x 256, 200 steps): gradient over forward time, and the
gradient checked against the FP64 tangent-linear oracle and central
differences; `accuracy` -- per-field relative L1
of the mixed step against the FP64 step after 1000 steps of the workload, and
one FP64 step (production and strict builds) against the oracle's first step
over every zone; `cpu_baseline` -- the oracle (the reference's step restated
in C, bit-identical to host builds of the reference kernels) on the host
cores over the whole workload, a bounded number of steps.

--impl reference times that CPU step on the same workload, set up with the
oracle's own metric tables, so no code of the CUDA library is loaded; it
reports the steps it actually ran (at most K, within --cpu-budget seconds).
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
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c3": dict(n1=384, n2=192, n3=192, rout=1000.0),
    "c2": dict(n1=192, n2=96, n3=64, rout=1000.0),
}


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def algorithmic_bytes_per_cell_update(n3: int) -> float:
    """Minimal FP64 traffic of one cell advanced one full RK2 step: half stage
    reads p^n (8) + ps^n (3), writes p* (8) + ps* (3) + U^n (6); full stage
    reads p* (8) + ps* (3) + ps^n (3) + U^n (6), writes p^{n+1} (8) +
    ps^{n+1} (3): 59 words; plus the axisymmetric metric (5 locations x 21 +
    40 connection = 145 words per (i, j) column) read once per sub-step."""
    return 59 * 8 + 2 * 1160.0 / n3


def kernel_bytes(slot: str, d: dict, width: float = 8.0) -> float:
    """Bytes one launch of a kernel group must move (FP64 storage; with width 4
    the fluxes and EMFs are float, as in the mixed-precision step):
    flux_d   per face: 9 primitives + 1 normal face field read, 9 fluxes written,
             plus the face metric (21 words) once per (i, j) column;
    update   (k_cons) per zone: 9 primitives, 9 cached conserved values and 27
             face fluxes read or written, 7 conserved values written, plus the
             centre metric and connection (61 words) per column;
    invert   per zone: 9 primitives (initial guess) + 7 conserved values + 3 face
             fields read, 9 primitives and 1 int flag written, plus the centre
             metric and face volumes (23 words) per column;
    emf_centre per zone (one ghost layer around): 3 velocities and 3 face
             fields read, 3 centre EMFs written;
    emf_edge   per edge: 3 centre EMFs and 9 face fluxes read, 3 EMFs written;
    face_update per face triple: 3 EMFs read, old and new face fields;
    update_invert (k_cons_tma with the primary inversion inside) per zone:
             the update's reads, 3 face fields read, 9 primitives and 1 int
             flag written, plus the update's metric; the 7 words of W and the
             inversion's guess never travel (the guess is the state the
             update read)."""
    n1, n2, n3 = d["n1"], d["n2"], d["n3"]
    if slot.startswith("flux"):
        k = int(slot[-1])
        nf = (n1 + 2 - (k == 1)) * (n2 + 2 - (k == 2)) * (n3 + 2 - (k == 3))
        ncol = (n1 + 2 - (k == 1)) * (n2 + 2 - (k == 2))
        return (10 * 8.0 + 9 * width) * nf + 21 * 8.0 * ncol
    if slot == "update":
        return (25 * 8.0 + 27 * width) * n1 * n2 * n3 + 61 * 8.0 * n1 * n2
    if slot == "invert":
        return (28 * 8.0 + 4) * n1 * n2 * n3 + 23 * 8.0 * n1 * n2
    if slot == "update_invert":
        return (30 * 8.0 + 27 * width + 4) * n1 * n2 * n3 + 61 * 8.0 * n1 * n2
    if slot == "emf_centre":
        return (6 * 8.0 + 3 * width) * (n1 + 2) * (n2 + 2) * (n3 + 2)
    if slot == "emf_edge":
        return 15 * width * (n1 + 1) * (n2 + 1) * (n3 + 1)
    if slot == "face_update":
        return (6 * 8.0 + 3 * width) * (n1 + 1) * (n2 + 1) * (n3 + 1)
    return 0.0


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per active zone of
# one launch, from single-launch ncu captures of each kernel on the 3-D torus
# 192 x 96 x 64 (profiles/k_*_torus_192x96x64.md; inputs larger than L2, caches
# flushed before the launch). Every kernel's traffic grows with the number of
# zones (plus a per-column metric term under 1 %), so a launch on another block
# moves these figures times its zones. flux1 and flux2 share the row kernel;
# flux3 includes the centre EMFs (computed by the x3 kernel on 3-D blocks);
# invert adds the fallback pass's 2.9 B; update_invert is the update kernel
# with the primary inversion inside (the default on 3-D blocks with
# n3 >= 32 and no floors or repair).
NCU_DRAM_BYTES_PER_ZONE = {
    "fp64": {"flux1": 219.3, "flux2": 219.3, "flux3": 296.5, "update": 457.1, "invert": 223.6,
             "update_invert": 509.2, "emf_edge": 123.7, "face_update": 54.7},
    "mixed": {"flux1": 134.2, "flux2": 134.2, "flux3": 136.7, "update": 315.4, "invert": 223.4,
              "update_invert": 388.6, "emf_edge": 58.6, "face_update": 40.6},
}

# what limits each kernel group, read from the same captures
KERNEL_LIMITER = {
    "flux1": "latency: PPM stencil loads (long scoreboard) and dependent FP chains",
    "flux2": "latency: PPM stencil loads (long scoreboard) and dependent FP chains",
    "flux3": "latency: dependent FP64/FP32 chains of the four flux evaluations per face (and the centre EMFs)",
    "update": "FP64 fixed-latency chains after TMA-staged operand loads",
    "invert": "FP64 dependent Newton iterations (FP64 pipe 45 % active)",
    "update_invert": "FP64 fixed-latency chains of the update's sums and the Newton iterations "
                     "(FP64 pipe 35-45 % active)",
    "emf_centre": "memory latency (long scoreboard)",
    "emf_edge": "memory latency (long scoreboard)",
    "face_update": "memory latency (long scoreboard)",
}


# the resource that binds each kernel group, with its utilisation in the
# same captures (profiles/: FP64 pipe or issue slots active, % of peak; for
# the latency-bound ones the long-scoreboard stalls per issued instruction)
KERNEL_BOUND = {
    "fp64": {"flux1": ("fp64", "sm__pipe_fp64_cycles_active %", 49.0),
             "flux2": ("fp64", "sm__pipe_fp64_cycles_active %", 49.0),
             "flux3": ("fp64", "sm__pipe_fp64_cycles_active %", 44.9),
             "update": ("latency", "long-scoreboard stalls / issue", 6.13),
             "invert": ("fp64", "sm__pipe_fp64_cycles_active %", 54.9),
             "update_invert": ("fp64", "sm__pipe_fp64_cycles_active %", 34.8),
             "emf_edge": ("latency", "long-scoreboard stalls / issue", 6.74),
             "face_update": ("latency", "long-scoreboard stalls / issue", 12.0)},
    "mixed": {"flux1": ("issue", "sm__issue_active %", 59.0),
              "flux2": ("issue", "sm__issue_active %", 59.0),
              "flux3": ("issue", "sm__issue_active %", 68.8),
              "update": ("latency", "long-scoreboard stalls / issue", 3.25),
              "invert": ("fp64", "sm__pipe_fp64_cycles_active %", 47.9),
              "update_invert": ("fp64", "sm__pipe_fp64_cycles_active %", 45.3),
              "emf_edge": ("issue", "sm__issue_active %", 61.1),
              "face_update": ("latency", "long-scoreboard stalls / issue", 12.7)},
}


def inversion_fused(slots: dict, d: dict) -> bool:
    """The 3-D update kernel with bulk-copy staging (n3 >= 32) runs the
    primary inversion itself unless floors or a repair are on; the invert
    slot then times only the fallback pass over failed zones, a few % of the
    update's time rather than about as much."""
    return d["n3"] >= 32 and slots.get("invert", 0.0) < 0.25 * slots.get("update", 0.0)


def kernel_rooflines(slots: dict, d: dict, prec: str, hbm: float) -> dict:
    """Per kernel group, per launch: algorithmic bytes, achieved GB/s over its
    live CUDA-event time (two launches per step), fraction of the HBM peak,
    DRAM traffic from the ncu capture scaled to this block, and the limiter."""
    width = 4.0 if prec == "mixed" else 8.0
    zones = d["n1"] * d["n2"] * d["n3"]
    tab = NCU_DRAM_BYTES_PER_ZONE.get("mixed" if prec == "mixed" else "fp64", {})
    # 3-D blocks: the centre EMFs come out of the x3 flux kernel (their slot
    # then times only its event pair)
    fused_ec = d["n3"] > 1 and slots.get("emf_centre", 0.0) < 0.05
    fused_inv = inversion_fused(slots, d)
    out = {}
    for slot, ms in slots.items():
        if (fused_ec and slot == "emf_centre") or (fused_inv and slot == "invert"):
            continue
        key = "update_invert" if fused_inv and slot == "update" else slot
        kb = kernel_bytes(key, d, width)
        if fused_ec and slot == "flux3":
            kb += kernel_bytes("emf_centre", d, width)
        if kb <= 0 or ms <= 0:
            continue
        gbs = 2 * kb / (ms * 1e-3) / 1e9
        out[slot] = {"ms_per_step": ms, "algorithmic_bytes": kb, "achieved_gbs": gbs, "frac": gbs / hbm,
                     "traffic": tab[key] * zones if key in tab else None,
                     "limiter": KERNEL_LIMITER.get(key)}
        bd = KERNEL_BOUND.get("mixed" if prec == "mixed" else "fp64", {}).get(key)
        if bd:
            out[slot].update(bound=bd[0], bound_metric=bd[1], bound_value=bd[2])
    return out


def launches_per_step(pb, fused_inv: bool = True) -> int:
    """Kernels one RK2 step launches (two sub-steps and the step-size
    finalisation), following the stage sequence of the library; with the
    inversion inside the update, its primary pass launches nothing."""
    dims = [n > 1 for n in (pb.n1, pb.n2, pb.n3)]
    per_stage = sum(dims)                       # face fluxes
    per_stage += pb.bc[1] == "pole_refl"        # polar flux fix
    per_stage += 1 if pb.n3 > 1 else 2          # edge EMFs (+ centre EMFs; in 3-D the x3 flux kernel makes them)
    per_stage += pb.bc[1] == "pole_trans"       # polar EMF average
    per_stage += 1 + 1 + (1 if fused_inv else 2)   # face update, conserved update, inversion (fallback pass)
    per_stage += sum(dims)                      # ghost fills
    return 2 * per_stage + 1


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


class OracleRun:
    """The oracle -- the C restatement of the reference step, bit-identical to
    the reference's own kernels run on the host -- holding one problem, with
    OpenMP over zones on the host cores. Used only as the CPU baseline and the
    parity check of the benchmark, never as the thing measured on the GPU."""

    def __init__(self, pb):
        from oracle import oracle as O
        self.O, self.pb = O, pb
        ob = O.Block(pb.n1, pb.n2, pb.n3, pb.ng, pb.ksize, pb.gsize)
        ob.arrays["p"][:] = pb.p
        ob.arrays["ps"][:] = pb.ps
        geo = O.Geometry(pb.geo.gsize, pb.geo.gcov, pb.geo.gcon, pb.geo.gdet, pb.geo.conn)
        self.s = O.Setup(ob, geo, pb.dx, pb.gam, pb.cour, 1, 1, (O.BC_OUTFLOW, O.BC_POLE_TRANS, O.BC_PERIODIC), 1)
        O.oracle_bound(self.s)
        self.threads = O.num_threads()

    def step(self, dt):
        O = self.O
        return O.step(lambda s_, f, Dt, d, c: O.oracle_stage(s_, f, Dt, d, c),
                      lambda s_, a, b: O.oracle_bound(s_, a, b), self.s, dt)

    def run(self, dt, steps, budget_s=None):
        """Up to `steps` RK2 steps with the CFL step-size rule; stops early
        once `budget_s` seconds have passed. Returns (steps run, seconds, dt)."""
        t0 = time.perf_counter()
        n = 0
        while n < steps:
            dt = min(self.step(dt), 1.3 * dt)
            n += 1
            if budget_s is not None and time.perf_counter() - t0 > budget_s:
                break
        return n, time.perf_counter() - t0, dt


def cpu_sample(pb, warmup: int, steps: int, budget_s: float):
    """Times the oracle on the whole workload: `warmup` untimed RK2 steps, then
    up to `steps` timed ones within `budget_s` seconds (the count actually run
    is reported). Returns (baseline dict, oracle run, step-1 state)."""
    orc = OracleRun(pb)
    dt0 = 0.2 * min(pb.dx[:2])
    dt = orc.step(dt0)   # the first step starts from dt0, like the GPU runs
    first = (orc.s.blk.arrays["p"].copy(), orc.s.blk.arrays["ps"].copy(), dt0)
    dt = min(dt, 1.3 * dt0)
    if warmup > 1:
        _, _, dt = orc.run(dt, warmup - 1)
    n, el, dt = orc.run(dt, steps, budget_s)
    cells = pb.n1 * pb.n2 * pb.n3
    cb = {"value": cells * n / el, "unit": "cell-updates/s", "cores": orc.threads, "kind": "port",
          "sample": f"the whole {pb.n1}x{pb.n2}x{pb.n3} torus, {n} timed RK2 step(s) after {max(1, warmup)} "
                    f"untimed, OpenMP over zones ({orc.threads} threads)",
          "steps": n, "ms_per_step": el * 1e3 / n}
    return cb, orc, first


def run_reference(args):
    """The reference's step on the host cores, on the same workload: the
    oracle (bit-identical to host builds of the reference kernels) with its
    own metric tables -- no code of the CUDA library is loaded."""
    rank, world, _ = _dist()
    if rank != 0:
        return
    from hamr_gamma_wind_b200 import problems
    from oracle import oracle as O
    wl = WORKLOADS[args.workload]
    pb = problems.fm_torus(wl["n1"], wl["n2"], wl["n3"], rout=wl["rout"], geometry=O.build_geometry)
    cb, _, _ = cpu_sample(pb, warmup=1, steps=args.steps, budget_s=args.cpu_budget)
    out = {"metric": "cell-updates/s", "value": cb["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
           "steps": cb["steps"], "warmup": 1, "requested_steps": args.steps, "requested_warmup": args.warmup,
           "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "impl": "reference",
           "dtype": "f64", "data": "synthetic", "vs_baseline": None, "scaling": "weak",
           "config": _config(wl, "fp64", args, same_config=True),
           "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "native_so_loaded": _loaded_native()}
    print(json.dumps(out), flush=True)


def _loaded_native():
    """Shared objects of this repository mapped into the process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if line.strip() else ""
                if path.endswith(".so") and path.startswith(ROOT):
                    out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def _config(wl, precision, args, **extra):
    return {"workload": f"3-D FM torus {wl['n1']}x{wl['n2']}x{wl['n3']} (a=0.9375, r_in=6, r_max=12, "
                        f"gamma=13/9, beta_min=100), {precision}",
            "zones": wl["n1"] * wl["n2"] * wl["n3"], "precision": precision, "recon": args.recon,
            "riemann": args.riemann, "floors": bool(args.floors), "repair": args.repair,
            "l2": "inputs larger than L2 (no flush)", "dt_update_interval": 16, **extra}


def _measure(pb, precision, args, stream, world, strict=False):
    """Device time of K RK2 steps of one block (after the warm-up) and the
    per-kernel-group breakdown; returns (ms, dt, blk). strict: the library
    build without multiply-add contraction (the one that reproduces the
    reference's roundings)."""
    import torch
    from hamr_gamma_wind_b200.api import Block
    blk = Block(**pb.block_kwargs(), precision=precision, stream=ctypes_stream(stream), recon=args.recon,
                riemann=args.riemann, floors=args.floors, repair=args.repair, strict=strict)
    blk.set_geometry(pb.geo)
    blk.upload(pb.p, pb.ps)
    blk.bound()
    dt = 0.2 * min(pb.dx[:2])
    # warm-up: W steps, then K more that capture the K-step graph the timed
    # region replays (a block caches one graph; capturing the W-step graph
    # last would put the K-step capture inside the timed region)
    dt = blk.step_ch(args.warmup, dt, interval=16)
    dt = blk.step_ch(args.steps, dt, interval=16)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        dt = blk.step_ch(args.steps, dt, interval=16)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    return ms, dt, blk, clk.summary()


def _kernel_profile(blk, dt):
    import ctypes
    from hamr_gamma_wind_b200 import _lib
    prof = np.zeros(len(_lib.PROF_SLOTS))
    blk._check(blk.L.hamr_profile_step(blk.ctx, dt, 2, prof.ctypes.data_as(ctypes.c_void_p), len(prof)),
               "hamr_profile_step")
    return dict(zip(_lib.PROF_SLOTS, prof.tolist()))


def run_ours(args):
    import ctypes
    import torch
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from hamr_gamma_wind_b200 import problems

    wl = WORKLOADS[args.workload]
    pb = problems.fm_torus(wl["n1"], wl["n2"], wl["n3"], rout=wl["rout"])
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    cells = pb.n1 * pb.n2 * pb.n3
    # fp64: the plain drop-in from the build that keeps the reference's
    # roundings (no multiply-add contraction: matches the oracle to the last
    # bits); fp64_fma: the same step from the contracted build; mixed: the
    # mixed-precision step (contracted build)
    variants = {"fp64": ("fp64", True), "fp64_fma": ("fp64", False), "mixed": ("mixed", False)}
    precs = ["fp64", "fp64_fma", "mixed"] if args.precision == "both" else [args.precision]
    runs = {}
    for prec in precs:
        ms, dt, blk, clocks = _measure(pb, variants[prec][0], args, stream, world, strict=variants[prec][1])
        runs[prec] = dict(ms=ms, value=world * cells * args.steps / (ms * 1e-3), clocks=clocks)
        if args.kernels_only:
            blk.close()
            continue
        if args.floors or args.repair != "none":
            # failure counters accumulated over every step run so far (2D,
            # 1dvsq2fix1, 1dfix1, floor gamma failure, repair without a stencil)
            runs[prec]["failures"] = blk.download_flags()[1].reshape(5, -1).sum(axis=1).tolist()
        runs[prec]["kernels"] = _kernel_profile(blk, dt)
        runs[prec]["dt"] = dt
        if prec == precs[-1]:
            head_blk = blk
        else:
            blk.close()
    head = precs[-1]
    value = runs[head]["value"]
    if args.kernels_only:
        if rank == 0:
            print(json.dumps({"metric": "cell-updates/s", "value": value, "ms_per_step": runs[head]["ms"] / args.steps,
                              "zones": cells, "precision": head, "note": "kernels only (profiling run)",
                              "runs": {k: {"value": v["value"]} for k, v in runs.items()}}), flush=True)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    blk = head_blk
    dt = runs[head]["dt"]
    slots = runs[head]["kernels"]
    top = max(slots, key=slots.get)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    width = 4.0 if head == "mixed" else 8.0
    kroof = kernel_rooflines(slots, wl, head, hbm)
    kb = kroof[top]["algorithmic_bytes"] if top in kroof else kernel_bytes(top, wl, width)
    achieved = kroof[top]["achieved_gbs"] if top in kroof else 0.0
    ms = runs[head]["ms"]
    step_gbs = algorithmic_bytes_per_cell_update(pb.n3) * cells / (ms * 1e-3 / args.steps) / 1e9

    # end to end through the public API with host buffers: upload from pinned
    # memory, one step, download of the new state, every step
    nk = 9 * blk.ksize
    hp = torch.empty(nk, dtype=torch.float64, pin_memory=True).numpy()
    hs = torch.empty(3 * blk.ksize, dtype=torch.float64, pin_memory=True).numpy()
    p_now, ps_now = blk.download()
    hp[:] = p_now
    hs[:] = ps_now
    n_e2e = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        blk.L.hamr_upload(blk.ctx, hp.ctypes.data_as(ctypes.c_void_p), hs.ctypes.data_as(ctypes.c_void_p))
        dt = min(blk.step(dt), 1.3 * dt)
        blk.L.hamr_download(blk.ctx, hp.ctypes.data_as(ctypes.c_void_p), hs.ctypes.data_as(ctypes.c_void_p))
    e2e_s = time.perf_counter() - t0
    e2e_val = world * cells * n_e2e / e2e_s
    bytes_io = (nk + 3 * blk.ksize) * 8
    p_end, _ = blk.download()
    finite = bool(np.isfinite(blk.active(p_end)).all())
    blk.close()

    # untimed blocks: a failure in one is reported in the line, not fatal
    accuracy = None
    if not args.no_accuracy and rank == 0:
        try:
            accuracy = _accuracy_block(pb, args, stream)
        except Exception as exc:
            accuracy = {"error": f"{type(exc).__name__}: {exc}"}
    adjoint = None
    if not args.no_adjoint and rank == 0:
        try:
            adjoint = _adjoint_block(args, fd_directions=8, tlm_directions=7)
        except Exception as exc:
            adjoint = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.set_stream(stream)
    cb = None
    if rank == 0:
        try:
            cb, orc, first = cpu_sample(pb, warmup=1, steps=2, budget_s=args.cpu_budget)
            if accuracy is not None and "error" not in accuracy:
                accuracy.update(_step1_vs_oracle(pb, first, stream))
        except Exception as exc:  # the oracle is test infrastructure; report, do not fail the bench
            cb = {"value": None, "error": str(exc)}

    if rank == 0:
        out = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else "f32 flux/EMF + f64 update/inversion", "data": "synthetic",
            "config": _config(wl, head, args, parallelism=f"replicas x{world}",
                              builds={"fp64": "libhamr_b200_strict.so (no multiply-add contraction)",
                                      "fp64_fma": "libhamr_b200.so", "mixed": "libhamr_b200.so"}),
            "precisions": {k: {"value": v["value"], "ms_per_step": v["ms"] / args.steps,
                               "kernel_ms_per_step": v.get("kernels"),
                               **({"failures": v["failures"]} if "failures" in v else {})}
                           for k, v in runs.items()},
            "gpu_launches": args.steps * launches_per_step(pb, inversion_fused(slots, wl)) + 1,
            "roofline": {"bound": "hbm", "kernel": ("update+invert" if top == "update" and inversion_fused(slots, wl)
                                                    else top),
                         "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": kroof.get(top, {}).get("traffic"),
                         "algorithmic_bytes": kb, "limiter": kroof.get(top, {}).get("limiter"),
                         "binding": {k: kroof.get(top, {}).get(k) for k in ("bound", "bound_metric", "bound_value")},
                         "traffic_source": "ncu DRAM bytes per zone, torus 192x96x64 capture, times zones",
                         "peak_source": peak_src},
            "kernel_rooflines": kroof,
            "step_roofline": {"algorithmic_bytes_per_cell_update": algorithmic_bytes_per_cell_update(pb.n3),
                              "achieved_gbs": step_gbs, "frac": step_gbs / hbm},
            "clocks": runs[head]["clocks"],
            "e2e": {"value": e2e_val, "unit": "cell-updates/s", "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io, "steps": n_e2e},
            "state_finite": finite,
        }
        if "fp64" in runs and "mixed" in runs:
            out["mixed_over_fp64"] = runs["mixed"]["value"] / runs["fp64"]["value"]
        if accuracy is not None:
            out["accuracy"] = accuracy
        if adjoint is not None:
            out["adjoint"] = adjoint
        out["cpu_baseline"] = cb
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def _rel_errs(a, b, names, l1=True):
    """Per-field relative L1 (or max) difference of a against b."""
    out = {}
    for k, n in enumerate(names):
        d, r = np.abs(a[k] - b[k]), np.abs(b[k])
        out[n] = float(d.sum() / max(r.sum(), 1e-300)) if l1 else float(d.max() / max(r.max(), 1e-300))
    return out


PRIM_NAMES = ["rho", "u", "u1", "u2", "u3", "B1", "B2", "B3"]
FACE_NAMES = ["face_B1", "face_B2", "face_B3"]


def _accuracy_block(pb, args, stream):
    """Per-field relative L1 difference of the mixed-precision step against
    the FP64 step (the build without contraction, which tracks the oracle)
    after `accuracy_steps` steps of the workload from the same initial state
    with the same step-size rule (device runs, untimed)."""
    from hamr_gamma_wind_b200.api import Block
    nsteps = args.accuracy or 1000
    out = {}
    for prec in ("fp64", "mixed"):
        blk = Block(**pb.block_kwargs(), precision=prec, stream=ctypes_stream(stream), strict=prec == "fp64")
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        dt = 0.2 * min(pb.dx[:2])
        left = nsteps
        while left > 0:
            n = min(left, 100)
            dt = blk.step_ch(n, dt, interval=16)
            left -= n
        p, ps = blk.download()
        out[prec] = (pb.active(p).copy(), pb.active(ps).copy(), dt)
        blk.close()
    p64, s64, dt64 = out["fp64"]
    p32, s32, dt32 = out["mixed"]
    errs = _rel_errs(p32, p64, PRIM_NAMES)
    errs.update(_rel_errs(s32, s64, FACE_NAMES))
    return {"steps": nsteps, "l1_rel_mixed_vs_fp64": errs, "target_rho_l1": 1e-5,
            "dt_after_fp64": dt64, "dt_after_mixed": dt32,
            "finite": bool(np.isfinite(p32).all() and np.isfinite(p64).all())}


def _step1_vs_oracle(pb, first, stream):
    """One FP64 step on the GPU from the workload's initial state against the
    oracle's first step (the reference's step, run on the host): the
    production build (fused multiply-adds) per field in relative L1 and max
    over all active zones, and the strict build (no contraction) in max."""
    from hamr_gamma_wind_b200.api import Block
    p_o, ps_o, dt0 = first
    po = pb.active(p_o)
    so = pb.active(ps_o)
    res = {}
    for strict in (False, True):
        blk = Block(**pb.block_kwargs(), precision="fp64", strict=strict, stream=ctypes_stream(stream))
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        blk.step(dt0)
        p, ps = blk.download()
        blk.close()
        pa, sa = pb.active(p), pb.active(ps)
        key = "strict_fp64_vs_oracle_step1" if strict else "fp64_vs_oracle_step1"
        res[key] = {"max_rel": {**_rel_errs(pa, po, PRIM_NAMES, l1=False), **_rel_errs(sa, so, FACE_NAMES, l1=False)}}
        if not strict:
            res[key]["l1_rel"] = {**_rel_errs(pa, po, PRIM_NAMES), **_rel_errs(sa, so, FACE_NAMES)}
    return res


ENSEMBLE = dict(count=64, nmin=32, nmax=96, seed=2024)


def run_ensemble(args):
    """Batched ensemble: 64 seeded magnetised tori of uneven sizes (each edge
    uniform in [32, 96]), spins uniform in [0, 0.99], r_max uniform in
    [10, 16], advanced together by hamr_batch_advance (one launch per phase
    for all members, captured CUDA graph) after hamr_batch_autotune. Reports
    ensemble cell-updates/s per precision, the same tile maps run as one
    persistent cooperative launch per sub-step (`persistent`), the same
    ensemble stepped member by member (each member's own captured graph, one
    after another on the same stream) for comparison, and the autotuner's
    choices."""
    import time
    import torch
    from hamr_gamma_wind_b200 import problems
    from hamr_gamma_wind_b200.api import Batch, Block
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if rank != 0:
        return
    pbs, draws = problems.torus_ensemble(**ENSEMBLE)
    cells = sum(pb.n1 * pb.n2 * pb.n3 for pb in pbs)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    cs = ctypes_stream(stream)
    precs = ["fp64", "mixed"] if args.precision == "both" else [args.precision.replace("fp64_fma", "fp64")]
    runs = {}
    for prec in precs:
        blocks = []
        for pb in pbs:
            b = Block(**pb.block_kwargs(), precision=prec, stream=cs)
            b.set_geometry(pb.geo)
            b.upload(pb.p, pb.ps)
            b.bound()
            blocks.append(b)
        batch = Batch(blocks, stream=cs)
        dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
        t0 = time.perf_counter()
        tun = batch.autotune(dts, reps=2)
        t_tune = time.perf_counter() - t0
        dts = batch.advance(args.steps, dts, interval=16)     # graph capture
        dts = batch.advance(args.warmup, dts, interval=16)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record(stream)
            dts = batch.advance(args.steps, dts, interval=16)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        # the same tile maps in one persistent cooperative launch per sub-step
        try:
            batch.set_persistent(True)
            dtp = batch.advance(args.steps, dts, interval=16)     # graph capture
            dtp = batch.advance(args.warmup, dtp, interval=16)
            torch.cuda.synchronize()
            e0.record(stream)
            dtp = batch.advance(args.steps, dtp, interval=16)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_p = e0.elapsed_time(e1)
            persistent = {"value": cells * args.steps / (ms_p * 1e-3), "ms_per_step": ms_p / args.steps}
            batch.set_persistent(False)
            dts = dtp
        except Exception as exc:
            persistent = {"error": f"{type(exc).__name__}: {exc}"}
        # member by member: each block's own graph, back to back
        dt1 = [b.step_ch(args.steps, d, interval=16) for b, d in zip(blocks, dts)]
        torch.cuda.synchronize()
        e0.record(stream)
        dt1 = [b.step_ch(args.steps, d, interval=16) for b, d in zip(blocks, dt1)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms_seq = e0.elapsed_time(e1)
        finite = all(bool(np.isfinite(b.active(b.download()[0])).all()) for b in blocks)
        runs[prec] = dict(value=cells * args.steps / (ms * 1e-3), ms_per_step=ms / args.steps,
                          unbatched_value=cells * args.steps / (ms_seq * 1e-3), persistent=persistent,
                          autotune_s=t_tune, tuning=tun, clocks=clk.summary(), finite=finite)
        batch.close()
        for b in blocks:
            b.close()
    head = precs[-1]
    out = {"metric": "cell-updates/s", "value": runs[head]["value"], "unit": "cell-updates/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": runs[head]["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if head == "fp64" else "f32 flux/EMF + f64 update/inversion", "data": "synthetic",
           "config": {"workload": f"ensemble of {len(pbs)} FM tori, edges U[{ENSEMBLE['nmin']},{ENSEMBLE['nmax']}], "
                                  f"a U[0,0.99], r_max U[10,16], seed {ENSEMBLE['seed']}", "zones": cells,
                      "precision": head, "members": [d["n"] for d in draws], "l2": "inputs larger than L2"},
           "precisions": {k: {kk: vv for kk, vv in v.items() if kk != "tuning"} for k, v in runs.items()},
           "tuning": {k: v["tuning"] for k, v in runs.items()},
           # per step: the phases that launch (tuned time > 0) in both
           # sub-steps and the step-size finalisation
           "gpu_launches": args.steps * (2 * sum(1 for v in runs[head]["tuning"].values() if v["ms"] > 0) + 1)}
    print(json.dumps(out), flush=True)


ADJOINT = dict(n=256, nsteps=200, every=20, directions=32, spin=0.9375, rout=40.0, generic=1e-3, radius=12.0)


def _adjoint_block(args, fd_directions, tlm_directions):
    """The adjoint workload: 2-D magnetised torus 256 x 256 (a = 0.9375,
    beta_min = 100, seeded tie-free perturbations), J = sum_n dt Mdot_n, the
    mass inflow through the sphere at the torus's pressure maximum r = 12
    integrated over 200 fixed-size steps; gradient w.r.t. the initial
    internal-energy field and gamma by hamr_adjoint_run (checkpoint every 20
    steps, recompute), timed against the forward sweep (hamr_mdot_forward),
    both on the build without contraction. Checked against the FP64
    tangent-linear oracle (the reference step on dual numbers, on the host)
    along `tlm_directions` seeded directions and gamma, and against central
    differences (relative steps 1e-6, 1e-7, 1e-8) along `fd_directions`."""
    import torch
    from hamr_gamma_wind_b200.api import Adjoint, Block
    from tests._adjoint import TorusRun, tangent_errors
    A = ADJOINT
    run = TorusRun(A["n"], A["n"], nsteps=A["nsteps"], every=A["every"], spin=A["spin"], rout=A["rout"],
                   strict=True, generic=A["generic"], radius=A["radius"])
    pb, dts = run.pb, run.dts
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    blk = Block(**pb.block_kwargs(), stream=ctypes_stream(stream), strict=True)
    blk.set_geometry(pb.geo)
    adj = Adjoint(blk, run.ih)

    def reset(u=None):
        q = pb.p.copy()
        if u is not None:
            pb.active(q)[1][:, :, 0] = u
        blk.upload(q, pb.ps)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(max(1, args.warmup)):
        reset(); adj.forward(dts)
    reset()
    torch.cuda.synchronize()
    e0.record(stream); J = adj.forward(dts); e1.record(stream); torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1)
    reset()
    adj.gradient(dts, A["every"])   # warm-up
    reset()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream); Jg, gp, gs, gg = adj.gradient(dts, A["every"]); e1.record(stream)
        torch.cuda.synchronize()
    t_run = e0.elapsed_time(e1)
    gu = pb.active(gp)[1][:, :, 0].copy()
    u0 = pb.active(pb.p)[1][:, :, 0].copy()

    def Ju(u):
        reset(u)
        return adj.forward(dts)
    rng = np.random.default_rng(2025)
    fd_steps = (1e-6, 1e-7, 1e-8)
    fd_errs = {e: [] for e in fd_steps}
    for _ in range(fd_directions):
        v = rng.standard_normal(u0.shape) * u0
        ad = float((gu * v).sum())
        for e in fd_steps:
            fd = (Ju(u0 + e * v) - Ju(u0 - e * v)) / (2 * e)
            fd_errs[e].append(abs(ad - fd) / max(abs(fd), 1e-300))
    adj.close()
    blk.close()
    t0 = time.perf_counter()
    tlm, tlm_g = tangent_errors(run, u0, pb.gam, gu, gg, ndir=tlm_directions) if tlm_directions else ([], None)
    t_tlm = time.perf_counter() - t0
    n = A["nsteps"]
    return {"workload": f"adjoint: 2-D FM torus {A['n']}x{A['n']} (a={A['spin']}, beta_min=100), J = sum_n dt Mdot "
                        f"through x1 face {run.ih} (r = {A['radius']}, the pressure maximum), {n} steps, "
                        f"checkpoint every {A['every']}",
            "adjoint_over_forward": t_run / t_fwd, "forward_ms_per_step": t_fwd / n,
            "gradient_ms_per_step": t_run / n, "J": J, "J_from_gradient_run": Jg, "dJ_dgamma": gg,
            "tangent_linear_check": {"directions": len(tlm), "reference": "oracle on forward-mode dual numbers (FP64)",
                                     "max_rel_err": float(np.max(tlm)) if len(tlm) else None,
                                     "median_rel_err": float(np.median(tlm)) if len(tlm) else None,
                                     "gamma_rel_err": tlm_g, "host_seconds": t_tlm},
            "fd_check": {"directions": fd_directions, "order": 2,
                         "by_rel_step": {f"{e:g}": {"max_rel_err": max(v) if v else None,
                                                     "median_rel_err": float(np.median(v)) if v else None}
                                         for e, v in fd_errs.items()}},
            "clocks": clk.summary()}


def run_adjoint(args):
    """The adjoint workload on its own line: metric adjoint/forward time."""
    import torch
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if rank != 0:
        return
    ndir = ADJOINT["directions"] if args.fd_directions is None else args.fd_directions
    r = _adjoint_block(args, ndir, tlm_directions=ndir)
    out = {"metric": "adjoint/forward time", "value": r["adjoint_over_forward"], "unit": "x", "n_gpus": 1,
           "steps": ADJOINT["nsteps"], "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": r["workload"], "zones": ADJOINT["n"] ** 2}, **r, "gpu_launches": None}
    print(json.dumps(out), flush=True)


def run_slabs(args):
    """The c3/c2 torus split along x1 (or x2, --slab-axis 2) into slabs
    (hamr_gamma_wind_b200.decomp):
    with one process, --slabs K slabs on one GPU swapping halos by device
    copies on one stream; under torchrun, one slab per rank, halos by NCCL
    point-to-point and the CFL minima by an all-reduce. Times the same K steps
    of the undivided block on rank 0 beside it (one process only). value =
    zones x steps / device time, max over ranks."""
    import torch
    from hamr_gamma_wind_b200 import decomp, problems
    from hamr_gamma_wind_b200.api import Block
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    wl = WORKLOADS[args.workload]
    prec = "mixed" if args.precision == "both" else args.precision.replace("fp64_fma", "fp64")
    pb = problems.fm_torus(wl["n1"], wl["n2"], wl["n3"], rout=wl["rout"])
    cells = pb.n1 * pb.n2 * pb.n3
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    cs = ctypes_stream(stream).value
    full = Block(**pb.block_kwargs(), precision=prec, stream=cs)
    full.set_geometry(pb.geo)
    full.upload(pb.p, pb.ps)
    full.bound()
    p0, ps0 = full.download()
    from dataclasses import replace
    pb = replace(pb, p=p0, ps=ps0)
    k = world if world > 1 else max(2, args.slabs)
    axis = args.slab_axis
    n = pb.n1 if axis == 1 else pb.n2
    widths = [n // k + (1 if r < n % k else 0) for r in range(k)]
    slabs = decomp.split(pb, widths, axis=axis)
    mine = [slabs[rank]] if world > 1 else slabs
    gs = decomp.gpu_slabs(mine, cs, precision=prec)
    ex = decomp.DistributedExchange(rank, world) if world > 1 else decomp.LocalExchange()
    st = decomp.SlabStepper(gs, ex, axis=axis)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(args.warmup):
        dt = min(st.step(dt), 1.3 * dt)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            dt = min(st.step(dt), 1.3 * dt)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    out = None
    if rank == 0:
        und = None
        if world == 1:
            d2 = 0.2 * min(pb.dx[:2])
            for _ in range(args.warmup):
                d2 = min(full.step(d2), 1.3 * d2)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                d2 = min(full.step(d2), 1.3 * d2)
            e1.record(stream)
            torch.cuda.synchronize()
            und = cells * args.steps / (e0.elapsed_time(e1) * 1e-3)
        out = {"metric": "cell-updates/s", "value": cells * args.steps / (ms * 1e-3), "unit": "cell-updates/s",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
               "dtype": "f64" if prec == "fp64" else "f32 flux/EMF + f64 update/inversion", "data": "synthetic",
               "config": {"workload": f"3-D FM torus {wl['n1']}x{wl['n2']}x{wl['n3']} split along x{axis} into {k} slabs "
                                      f"{widths}", "zones": cells, "precision": prec,
                          "exchange": "nccl" if world > 1 else "device copies, one stream",
                          "parallelism": f"x{axis} slabs x{k}"},
               "undivided_value_same_steps": und, "clocks": clk.summary(), "gpu_launches": None}
        print(json.dumps(out), flush=True)
    for g in gs:
        g.block.close()
    full.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=list(WORKLOADS) + ["c4", "c5"])
    ap.add_argument("--precision", default="both", choices=["fp64", "fp64_fma", "mixed", "both"])
    ap.add_argument("--fd-directions", type=int, default=None,
                    help="c5: finite-difference directions checked after the timing (default 32)")
    ap.add_argument("--recon", default="ppm", choices=["ppm", "mc"],
                    help="reconstruction of the c3/c2 torus (PPM as shipped, or MC)")
    ap.add_argument("--riemann", default="hll", choices=["hll", "hllc", "hlld"],
                    help="Riemann solver of the c3/c2 torus (HLL as shipped, HLLC or HLLD)")
    ap.add_argument("--floors", action="store_true",
                    help="c3/c2 torus with the opt-in drift-frame floors (off in the reference's step)")
    ap.add_argument("--repair", default="none", choices=["none", "reset", "neighbours"],
                    help="c3/c2 torus: repair of failed zones (none, as the reference's step)")
    ap.add_argument("--accuracy", type=int, default=0,
                    help="steps of the accuracy block (mixed vs FP64 per-field L1; default 1000)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the accuracy block (mixed vs FP64 after 1000 steps, step 1 vs the oracle)")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint block (C5 adjoint/forward time, tangent-linear and FD checks)")
    ap.add_argument("--cpu-budget", type=float, default=120.0,
                    help="seconds of timed oracle steps at most (CPU baseline and the reference arm)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="warm-up and timed steps only (for profiler runs)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="c3/c2 split into slabs: K slabs on one GPU, or one slab per rank under torchrun")
    ap.add_argument("--slab-axis", type=int, default=1, choices=[1, 2], help="split along x1 or x2")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c4":
        run_ensemble(args)
    elif args.workload == "c5":
        run_adjoint(args)
    elif args.slabs:
        run_slabs(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
