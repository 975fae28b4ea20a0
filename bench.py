"""Benchmark of the quasi-static slice loop on B200.

Workload (default): the nonlinear blowout wake, plain FP64 — 255 x 255 transverse cells over
[-6, 6]^2, 256 slices over zeta in [-8, 4], 65k plasma particles (1 per cell), a Gaussian driver
of 1e6 seeded macro-particles (sigma 0.3, 0.3, 1.0; peak density 10; gamma 2000; normalized
emittance 0.01), explicit Bx/By solver with multigrid, dt = 20. A "step" is one time step: the
full slice march (256 slices) including the FP64 beam push.

Metric: slices/s (whole job). `value` is device-timed (CUDA events on the library's stream,
beam already resident). `e2e` is timed through the public C ABI with the step's inputs (the
beam particles) uploaded from pinned host memory and the results (the pushed beam) read back
every step. `roofline` is computed live from per-kernel events of a profiled pass over the same
steps; `cpu_baseline` times this build's FP64 CPU oracle (oracle/, the reference itself cannot be
built here) on a bounded sample.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--config NAME]
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# algorithmic bytes per plasma particle per slice, FP64, explicit path (reads and writes of the
# particle arrays by deposit, explicit deposit and push): 21*8 + 24
BYTES_PER_PARTICLE_SLICE = {8: 21 * 8 + 24, 4: 21 * 4 + 24}
# plasma push alone: reads x_prev, y_prev, ux_h, uy_h, psi_h (+ valid byte), writes 10 reals
PUSH_BYTES = {8: 5 * 8 + 1 + 10 * 8, 4: 5 * 4 + 1 + 10 * 4}
# multigrid (the persistent solve, one launch per slice): per V-cycle (4/3) x (rhs 2 + coefficient
# 1 + solution 2 read + 2 written + residual 2) reals per level-0 point, plus one such pass for
# the first smoothing
MG_REALS_PER_POINT_VCYCLE = 4.0 / 3.0 * 9.0
MG_REALS_PER_POINT_FIRST = 9.0
# DRAM bytes (read 2 936 064 + write 0) of one k_mg_solve launch of the current kernel (two
# coarse-level blocks) from ncu (blowout_255, FP64, one launch after 300, `--set full`,
# profiles/k_mg_solve_blowout_255_fp64.md): the level-0 arrays stay in L2, so DRAM traffic is far
# below the algorithmic bytes
MG_NCU_DRAM_BYTES_FP64_255 = 2936064


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="blowout_255")
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--no-graphs", action="store_true")
    p.add_argument("--cpu-sample-steps", type=int, default=2,
                   help="whole steps of the FP64 CPU oracle timed for cpu_baseline")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    p.add_argument("--scale-config", default="channel_1023",
                   help="larger workload timed for FP64 vs mixed (one step each); '' to skip")
    p.add_argument("--adjoint-config", default="beam_loading_255",
                   help="workload of the adjoint timing (time per gradient); '' to skip")
    p.add_argument("--large-config", default="large_2047",
                   help="largest workload: one mixed-precision step and one adjoint gradient; '' to skip")
    return p.parse_args()


def job_rate(local_secs, units_per_rank, world, reduce_max):
    """Whole-job throughput of `world` independent replicas: the units of all ranks over the
    slowest rank's time (reduce_max takes the maximum over ranks; every rank must call it).
    Returns (units per second, that time)."""
    secs = reduce_max(local_secs)
    return units_per_rank * world / secs, secs


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def peaks():
    try:
        d = json.load(open(PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def workload_config(args, grid, n_plasma, n_beam, world):
    """The `config` object of both arms (the same dict, so that the two lines compare)."""
    return {"workload": args.config, "grid": [int(v) for v in grid], "plasma_particles": int(n_plasma),
            "beam_particles": int(n_beam), "solver": "explicit+multigrid", "precision": args.precision,
            "steps_timed": "whole steps (all slices, beam push included)",
            "parallelism": f"replicas{world}", "l2": "inputs larger than L2 per step (beam store)"}


def make_sim(text, precision, graphs):
    import hipace2_b200 as hp
    sim = hp.Hipace(text, precision=hp.MIXED if precision == "mixed" else hp.PLAIN_FP64, graphs=graphs)
    sim.init_data()
    return sim


def time_device_steps(sim, first, k, torch):
    stream = torch.cuda.ExternalStream(sim.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    sim.synchronize()
    e0.record(stream)
    for s in range(first, first + k):
        sim.step(s)
    e1.record(stream)
    sim.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def run_ours(args):
    import numpy as np
    import torch

    import hipace2_b200 as hp
    from cases import config

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    text = config(args.config)
    sim = make_sim(text, args.precision, graphs=not args.no_graphs)
    nx, ny, nz = sim.n_cell
    n_plasma = sim.get_plasma(0)["x"].size
    w = args.warmup
    k = args.steps
    n_beam0 = int(sim.get_beam(0)["x"].size)
    for s in range(w):
        sim.step(s)
    beam_w = sim.get_beam(0)  # state entering step w (input of the e2e leg)
    # ---- device-timed region (replicas: each rank runs its own independent simulation)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    l_before = sim.counters()["kernel_launches"]
    with ClockSampler(local) as clk:
        secs = time_device_steps(sim, w, k, torch)
    launches_in_timed = sim.counters()["kernel_launches"] - l_before

    def reduce_max(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    value, secs = job_rate(secs, nz * k, world, reduce_max)
    # ---- end to end through the C ABI with host buffers, on the same step indices and the same
    # initial beam as the device-timed region: a second simulation of the same deck runs the same
    # warm-up steps, then every timed step uploads its beam from pinned host memory, runs, and
    # reads the pushed beam back into pinned memory, which is the next step's input
    e2e_value, h2d, d2h = e2e_steps(text, args, beam_w, w, k, world, reduce_max, torch)
    # ---- profiled pass (kernel launches with events) for the roofline of the dominant kernel
    sim.set_profiling(True)
    for s in range(w + k, w + 2 * k):
        sim.step(s)
    classes = ["plasma_deposit", "beam_deposit", "poisson_psi_ez_bz", "explicit_deposit", "multigrid",
               "plasma_push", "beam_push", "beam_partition"]
    prof = {c: sim.profile(c) for c in classes}
    sim.set_profiling(False)
    total_prof = sum(v[0] for v in prof.values())
    dominant = max(prof, key=lambda c: prof[c][0])
    elem = 8 if args.precision == "fp64" else 4
    push_ms, push_n = prof["plasma_push"]
    peak, peak_kind = peaks()
    push_bytes = n_plasma * PUSH_BYTES[elem]
    achieved = push_bytes / (push_ms / 1e3 / max(push_n, 1)) / 1e9 if push_n else 0.0
    counters = sim.counters()
    # dominant kernel: the persistent multigrid solve (one launch per slice)
    mg_ms, mg_n = prof["multigrid"]
    vc = counters["mg_vcycles"] / max(counters["slices"], 1)
    mg_bytes = (vc * MG_REALS_PER_POINT_VCYCLE + MG_REALS_PER_POINT_FIRST) * nx * ny * elem
    mg_launch_ms = mg_ms / max(mg_n, 1)
    mg_achieved = mg_bytes / (mg_launch_ms / 1e3) / 1e9 if mg_n else 0.0
    line = {
        "metric": "slices/s",
        "value": value,
        "unit": "slices/s",
        "n_gpus": world,
        "steps": k,
        "warmup": w,
        "ms_per_step": secs / k * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 (beam f64)",
        "data": "synthetic: seeded Gaussian driver beam (Philox), lattice plasma",
        "config": workload_config(args, (nx, ny, nz), n_plasma, n_beam0, world),
        "graphs": not args.no_graphs,
        "particle_updates_per_s": n_plasma * nz * k * world / secs,
        "e2e": {"value": e2e_value, "unit": "slices/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": None,
        "roofline": {"bound": "hbm", "kernel": "k_mg_solve", "achieved": mg_achieved, "peak": peak,
                     "unit": "GB/s", "frac": mg_achieved / peak, "peak_kind": peak_kind,
                     "traffic": (MG_NCU_DRAM_BYTES_FP64_255
                                 if (args.config == "blowout_255" and elem == 8) else None),
                     "bytes_per_launch": mg_bytes, "launch_ms": mg_launch_ms,
                     "vcycles_per_launch": vc,
                     "note": "latency-bound: level-0 arrays live in L2; traffic from ncu, one cold launch"},
        "roofline_plasma_push": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "bytes_per_launch": push_bytes,
                                 "launch_ms": push_ms / max(push_n, 1)},
        "kernel_share": {c: (prof[c][0] / total_prof if total_prof else 0) for c in classes},
        "dominant_kernel_class": dominant,
        "mg_vcycles_per_slice": counters["mg_vcycles"] / max(counters["slices"], 1),
        "clocks": clk.summary(),
    }
    if rank == 0:
        line["gpu_launches"] = launches_in_timed
        if not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(text, args)
    sim.close()
    if rank == 0 and not args.no_mixed and args.precision == "fp64":
        line["mixed"] = mixed_vs_fp64(text, args, torch)
        if args.scale_config:
            line["scale_point"] = scale_point(args.scale_config, torch)
    if rank == 0 and args.adjoint_config and args.precision == "fp64":
        line["adjoint"] = adjoint_point(args.adjoint_config, torch)
        line["salame_vs_adjoint"] = salame_vs_adjoint(args.adjoint_config)
    if rank == 0 and args.precision == "fp64" and args.config == "blowout_255" and not args.no_mixed:
        line["linear_wake_64"] = linear_wake_point(torch, args.no_cpu)
        if args.large_config:
            line["large"] = large_point(args.large_config, torch)
    if rank == 0:
        print(json.dumps(line))
    sim.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def e2e_steps(text, args, beam_w, w, k, world, reduce_max, torch):
    """Steps w .. w+k-1 through the public C ABI with host buffers: a fresh simulation of the same
    deck runs the warm-up steps 0 .. w-1 (untimed), then each timed step uploads its input beam
    from pinned host memory (hpq_set_beam), runs (hpq_step) and reads the pushed beam back into
    pinned memory (hpq_get_beam), which becomes the next step's input. The first timed step's
    input is `beam_w`, the beam the device-timed run entered step w with, so both legs do the same
    work. Returns (slices/s of the job, H2D bytes per step, D2H bytes per step)."""
    import numpy as np
    sim = make_sim(text, args.precision, graphs=not args.no_graphs)
    nz = sim.n_cell[2]
    for s in range(w):
        sim.step(s)
    cap = beam_w["x"].size
    keys = ("x", "y", "z", "w", "ux", "uy", "uz", "id")

    def pinned_set():
        out = {}
        for key in keys:
            t = torch.empty(cap, dtype=torch.int64 if key == "id" else torch.float64).pin_memory()
            out[key] = t.numpy()
        return out

    bufs = [pinned_set(), pinned_set()]
    for key in keys:
        bufs[0][key][:] = beam_w[key]
    cur = {key: bufs[0][key][:cap] for key in keys}
    h2d = d2h = 0
    torch.cuda.synchronize()
    sim.synchronize()
    t0 = time.perf_counter()
    for i, s in enumerate(range(w, w + k)):
        n_in = cur["x"].size
        sim.set_beam(0, cur)
        sim.step(s)
        cur = sim.get_beam(0, out=bufs[(i + 1) % 2])
        h2d += n_in * (7 * 8 + 8)                 # 7 attributes + id
        d2h += cur["x"].size * (7 * 8 + 8 + 1)   # 7 attributes + id + validity flag
    sim.synchronize()
    secs = time.perf_counter() - t0
    sim.close()
    value, _ = job_rate(secs, nz * k, world, reduce_max)
    return value, h2d // k, d2h // k


def make_sim_env(text, precision, env=None, deterministic=False):
    """make_sim with environment switches read by the library at set-up (HPQ_DST, HPQ_MG_REFINE)."""
    import hipace2_b200 as hp
    env = env or {}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        sim = hp.Hipace(text, precision=hp.MIXED if precision == "mixed" else hp.PLAIN_FP64, graphs=True,
                        deterministic=deterministic)
        sim.init_data()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return sim


def rel_l2(a, b):
    import numpy as np
    n = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / n if n > 0 else float(np.linalg.norm(a - b))


def beam_moment_errors(m, d):
    """Per-slice beam centroid and normalized emittance of two in-situ records (a run and its FP64
    reference; BeamParticleContainer.cpp:476-548 moments): the centroid error as the weighted L2
    of the centroid difference over the weighted L2 of the rms size, the emittance error as a
    relative weighted L2, over the slices holding particles; and the projected emittance error."""
    import numpy as np
    out = {}
    w = d["sum(w)"]
    sel = w > 0
    for ax, u in (("x", "ux"), ("y", "uy")):
        def emit(r):
            vx = r["[%s^2]" % ax] - r["[%s]" % ax] ** 2
            vu = r["[%s^2]" % u] - r["[%s]" % u] ** 2
            cx = r["[%s*%s]" % (ax, u)] - r["[%s]" % ax] * r["[%s]" % u]
            return np.sqrt(np.maximum(vx * vu - cx * cx, 0.0)), np.sqrt(np.maximum(vx, 0.0))
        em, sm = emit(m)
        ed, sd = emit(d)
        ww = w[sel]
        out["centroid_%s_err_over_rms_size" % ax] = float(
            np.sqrt(np.sum(ww * (m["[%s]" % ax][sel] - d["[%s]" % ax][sel]) ** 2) / np.sum(ww * sd[sel] ** 2)))
        out["emittance_%s_rel_l2" % ax] = float(np.sqrt(np.sum(ww * (em[sel] - ed[sel]) ** 2) / np.sum(ww * ed[sel] ** 2)))

        def proj(r):
            t = r["sum"]
            names = hp_insitu_names()
            g = {k: t[i] for i, k in enumerate(names)}
            vx = g["[%s^2]" % ax] - g["[%s]" % ax] ** 2
            vu = g["[%s^2]" % u] - g["[%s]" % u] ** 2
            cx = g["[%s*%s]" % (ax, u)] - g["[%s]" % ax] * g["[%s]" % u]
            return np.sqrt(max(vx * vu - cx * cx, 0.0))
        pm, pd = proj(m), proj(d)
        out["projected_emittance_%s_rel" % ax] = abs(pm - pd) / pd if pd > 0 else None
    return out


def hp_insitu_names():
    import hipace2_b200 as hp
    return hp.INSITU_BEAM


def precision_errors(text, precision, beam, comps, env=None, deterministic=False, ref=None, steps=2):
    """Fields of step 0 and the beam moments entering step 1 (after one push) of one run, and
    their errors against `ref` (an earlier result of this function) when given."""
    sim = make_sim_env(text, precision, env, deterministic)
    sim.set_beam(0, beam)
    sim.set_diag(comps)
    sim.step(0)
    fields = {c: sim.get_diag(c) for c in comps}
    sim.step(1)
    moments = sim.get_insitu("beam")
    sim.close()
    res = {"fields": fields, "moments": moments}
    if ref is not None:
        err = {c + "_rel_l2": rel_l2(fields[c], ref["fields"][c]) for c in comps}
        err.update(beam_moment_errors(moments, ref["moments"]))
        res["errors"] = err
    return res


def mixed_vs_fp64(text, args, torch):
    """The same workload in mixed precision (FP32 plasma, fields and multigrid; FP64 beam) against
    the FP64 path on identical inputs: throughput, the relative L2 error of Ez, Psi, jz_beam and
    Bx over every slice of step 0, and the beam's per-slice centroid and emittance entering step
    1 (after one push in the mixed fields). The FP64 GPU path stands in for the FP64 oracle (it
    matches the oracle to <= 1e-10 over a whole step of this workload in the parity tests).
    Beside it: the FP64 noise floor (FP64 with floating-point atomics against FP64 in
    deterministic mode, and FP64 with the beam's x displaced by 1e-7 of its rms size), and the
    mixed path with one stage changed (the TF32x3 tensor-core DST instead of the FP32 FFT; FP64
    residual refinement of the multigrid), and a weak-wake version of the workload (the driver's
    weights scaled to a peak density of 0.5), where the plasma response is closer to linear."""
    import numpy as np
    comps = ["Ez", "Psi", "jz_beam", "Bx"]
    out = {}
    ref = make_sim(text, "fp64", graphs=True)
    beam = ref.get_beam(0)
    ref.close()
    mix = make_sim(text, "mixed", graphs=True)
    mix.set_beam(0, beam)
    nz = mix.n_cell[2]
    # speed: warm-up steps then timed steps, like the FP64 headline
    w, k = max(1, args.warmup), max(1, args.steps)
    for s in range(w):
        mix.step(s)
    secs = time_device_steps(mix, w, k, torch)
    mix.close()
    out["value"] = nz * k / secs
    out["unit"] = "slices/s"
    out["ms_per_step"] = secs / k * 1e3
    tdiag = text + "\nbeams.insitu_period = 1\n"
    d64 = precision_errors(tdiag, "fp64", beam, comps, deterministic=True)
    out.update(precision_errors(tdiag, "mixed", beam, comps, ref=d64)["errors"])
    out["error_reference"] = ("FP64 GPU path in deterministic mode, same beam: fields of step 0 (all slices), "
                              "beam moments entering step 1")
    out["dtype"] = "f32 plasma/fields/multigrid, f64 beam"
    floor = {}
    floor["fp64_atomics_vs_deterministic"] = precision_errors(tdiag, "fp64", beam, comps, ref=d64)["errors"]
    shifted = dict(beam)
    shifted["x"] = beam["x"] + 1e-7 * float(np.std(beam["x"]))
    floor["fp64_beam_x_displaced_1e-7_rms"] = precision_errors(tdiag, "fp64", shifted, comps, deterministic=True,
                                                              ref=d64)["errors"]
    out["fp64_noise_floor"] = floor
    abl = {}
    for name, env in (("tf32x3_tensor_core_dst", {"HPQ_DST": "tc"}), ("bf16x3_tensor_core_dst", {"HPQ_DST": "tc_bf16"}),
                      ("fp64_multigrid_refinement", {"HPQ_MG_REFINE": "1"})):
        r = precision_errors(tdiag, "mixed", beam, comps, env=env, ref=d64)["errors"]
        sim = make_sim_env(text, "mixed", env)
        sim.set_beam(0, beam)
        sim.step(0)
        r["slices_per_s"] = nz / time_device_steps(sim, 1, 1, torch)
        sim.close()
        abl[name] = r
    out["ablation"] = abl
    # weak wake: the same particles with weights scaled to a peak density of 0.5
    weak = tdiag
    wbeam = dict(beam)
    wbeam["w"] = beam["w"] * (0.5 / 10.0)
    w64 = precision_errors(weak, "fp64", wbeam, comps, deterministic=True)
    out["weak_wake"] = {"driver_density": 0.5,
                        "mixed": precision_errors(weak, "mixed", wbeam, comps, ref=w64)["errors"],
                        "fp64_atomics_vs_deterministic": precision_errors(weak, "fp64", wbeam, comps, ref=w64)["errors"]}
    return out


def scale_point(name, torch, sample_every=64):
    """The larger workload over its configured 5 steps in FP64 and in mixed precision: steps 1-3
    device-timed, steps 0 and 4 run slice by slice with every `sample_every`-th slice's fields
    read back (a full 3-D diagnostic would be 8 GB per component), and the mixed error against
    the FP64 GPU path on identical inputs for both; plus the FP64 noise floor of step 0 (FP64
    with floating-point atomics against FP64 in deterministic mode)."""
    import numpy as np
    from cases import config
    text = config(name)
    res = {"workload": name}
    comps = ["Ez", "Psi", "jz_beam", "Bx"]
    samples = {}
    beam = None

    def sampled_step(sim, step):
        got = {c: [] for c in comps}
        sim.begin_step(step)
        for s in range(sim.n_cell[2] - 1, -1, -1):
            sim.solve_one_slice(s)
            if s % sample_every == 0:
                for c in comps:
                    got[c].append(sim.get_field(c))
        sim.end_step()
        return {c: np.array(v) for c, v in got.items()}

    for prec, det in (("fp64", True), ("fp64", False), ("mixed", False)):
        sim = make_sim_env(text, prec, deterministic=det)
        if beam is None:
            beam = sim.get_beam(0)
        else:
            sim.set_beam(0, beam)
        nz = sim.n_cell[2]
        key = prec + ("_det" if det else "")
        first = sampled_step(sim, 0)
        if det:
            samples[key] = {0: first}
            sim.close()
            continue
        secs = time_device_steps(sim, 1, 3, torch)
        last = sampled_step(sim, 4)
        samples[key] = {0: first, 4: last}
        res[prec + "_slices_per_s"] = 3 * nz / secs
        res[prec + "_ms_per_step"] = secs / 3 * 1e3
        if prec == "fp64":
            res["grid"] = sim.n_cell
            res["plasma_particles"] = int(sim.get_plasma(0)["x"].size)
        sim.close()
    res["mixed_speedup"] = res["mixed_slices_per_s"] / res["fp64_slices_per_s"]
    for step in (0, 4):
        for c in comps:
            res["step%d_%s_rel_l2" % (step, c)] = rel_l2(samples["mixed"][step][c], samples["fp64"][step][c])
    res["fp64_noise_floor_step0"] = {c + "_rel_l2": rel_l2(samples["fp64"][0][c], samples["fp64_det"][0][c])
                                     for c in comps}
    res["steps"] = "5 (0-4): steps 1-3 timed, steps 0 and 4 sampled"
    res["error_reference"] = "FP64 GPU path, same beam, every %d-th slice of steps 0 and 4" % sample_every
    return res


def linear_wake_point(torch, no_cpu=False):
    """The CPU-runnable workload (64 x 64 x 100, predictor-corrector Bx/By with 3 iterations, 1e5
    driver particles): all 11 steps (0-10) on the GPU in FP64 (device time) and, unless skipped,
    in the FP64 CPU oracle on the same seeded beam (all host threads)."""
    from cases import config
    text = config("linear_wake_64")
    sim = make_sim(text, "fp64", graphs=True)
    nz = sim.n_cell[2]
    sim.step(0)  # graph capture and warm-up (step 0 again below on a fresh simulation)
    sim.close()
    sim = make_sim(text, "fp64", graphs=True)
    secs = time_device_steps(sim, 0, 11, torch)
    sim.close()
    res = {"workload": "linear_wake_64", "grid": [64, 64, nz], "steps": 11, "gpu_slices_per_s": 11 * nz / secs,
           "gpu_ms_per_step": secs / 11 * 1e3}
    if not no_cpu:
        o, dt = oracle_run(text, 0, 11)
        res["cpu_oracle_slices_per_s"] = 11 * nz / dt
        res["cpu_oracle_threads"] = o.L.oracle_threads()
        res["gpu_over_cpu"] = res["gpu_slices_per_s"] / res["cpu_oracle_slices_per_s"]
    return res


def large_point(name, torch):
    """The largest workload (2047 x 2047 x 2048, 4.2M plasma particles, 1.2e7 beam particles): one
    mixed-precision step (device time) and one adjoint gradient with its forward (FP64, wall time
    between device synchronisations), with the device memory in use."""
    import numpy as np
    import hipace2_b200 as hp
    from cases import adjoint_knots, config
    text = config(name)
    res = {"workload": name, "grid": [int(v) for v in _n_cell(text)]}
    sim = make_sim(text, "mixed", graphs=True)
    nz = sim.n_cell[2]
    sim.step(0)
    secs = time_device_steps(sim, 1, 1, torch)
    res["mixed_slices_per_s"] = nz / secs
    res["mixed_ms_per_step"] = secs * 1e3
    sim.close()
    sim = hp.Hipace(text, graphs=True)
    sim.init_data()
    theta = adjoint_knots(n_profile=int(_key(text, "adjoint.n_profile_knots")),
                          n_density=int(_key(text, "adjoint.n_density_knots")))
    sim.adjoint(theta, grad=False)  # allocation of the records and checkpoints, graph capture
    sim.synchronize()
    t0 = time.perf_counter()
    sim.adjoint(theta, grad=False)
    sim.synchronize()
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    J, g = sim.adjoint(theta)
    sim.synchronize()
    t_grad = time.perf_counter() - t0
    free, total = torch.cuda.mem_get_info()
    sim.close()
    res.update({"adjoint_seconds_forward": t_fwd, "adjoint_seconds_per_gradient": t_grad,
                "gradient_over_forward": t_grad / t_fwd, "adjoint_dtype": "f64",
                "device_memory_in_use_gb_at_gradient": (total - free) / 1e9,
                "objective": J, "max_abs_grad": float(np.abs(g).max()),
                "checkpoint_interval": int(_key(text, "adjoint.checkpoint_interval"))})
    return res


def adjoint_point(name, torch, reps=3):
    """Adjoint of one step (hpq_adjoint_grad) on the beam-loading workload: device-synchronised
    wall time per gradient (forward with checkpoints, recomputation, reverse sweep), per forward
    of the same step (no reverse) and per plain step (hpq_step, beam push included), plus a
    central-difference check of 8 seeded witness-profile knots (FP64 forward, step 1e-4
    relative)."""
    import numpy as np
    import hipace2_b200 as hp
    from cases import adjoint_knots, config
    text = config(name)
    sim = hp.Hipace(text, graphs=True)
    sim.init_data()
    nz = sim.n_cell[2]
    n_profile = int(_key(text, "adjoint.n_profile_knots"))
    n_density = int(_key(text, "adjoint.n_density_knots"))
    theta = adjoint_knots(n_profile=n_profile, n_density=n_density)

    def timed(f, n, s=sim):
        f()
        s.synchronize()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            r = f()
        s.synchronize()
        return (time.perf_counter() - t0) / n, r

    t_fwd, J = timed(lambda: sim.adjoint(theta, grad=False), reps)
    t_grad, (J2, g) = timed(lambda: sim.adjoint(theta), reps)
    fd = {}
    scale = float(np.abs(g).max())
    picks = np.random.default_rng(2024).choice(np.arange(4, n_profile - 4), size=8, replace=False)
    for k in sorted(int(v) for v in picks):
        h = 1e-4 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        d = (sim.adjoint(tp, grad=False) - sim.adjoint(tm, grad=False)) / (2 * h)
        fd[str(k)] = {"adjoint": float(g[k]), "central_difference": d,
                      "err_rel_to_max_grad": abs(float(g[k]) - d) / scale}
    step = [0]

    def plain():
        sim.step(step[0])
        step[0] += 1

    t_step, _ = timed(plain, 2)
    sim.close()
    # the same gradient with the single-precision forward (FP64 reverse sweep), same beams
    mix = hp.Hipace(text, precision=hp.MIXED, graphs=True)
    mix.init_data()
    tm_fwd, Jm = timed(lambda: mix.adjoint(theta, grad=False), reps, mix)
    tm_grad, (Jm2, gm) = timed(lambda: mix.adjoint(theta), reps, mix)
    mstep = [0]

    def mplain():
        mix.step(mstep[0])
        mstep[0] += 1

    tm_step, _ = timed(mplain, 2, mix)
    mix.close()
    mixed = {"seconds_per_gradient": tm_grad, "seconds_forward": tm_fwd, "seconds_plain_step": tm_step,
             "gradient_over_forward": tm_grad / tm_fwd, "gradient_over_plain_step": tm_grad / tm_step,
             "objective_rel_diff_from_f64": abs(Jm - J) / abs(J),
             "grad_max_abs_diff_over_max_grad": float(np.abs(gm - g).max()) / scale,
             "grad_rel_l2_from_f64": float(np.linalg.norm(gm - g) / np.linalg.norm(g)),
             "dtype": "f32 forward (beam f64), f64 reverse"}
    return {"workload": name, "grid": [int(v) for v in _n_cell(text)], "params": int(theta.size),
            "checkpoint_interval": int(_key(text, "adjoint.checkpoint_interval")),
            "seconds_per_gradient": t_grad, "seconds_forward": t_fwd, "seconds_plain_step": t_step,
            "gradient_over_plain_step": t_grad / t_step, "gradient_over_forward": t_grad / t_fwd,
            "objective": J, "max_abs_grad": scale, "fd_check": fd, "dtype": "f64",
            "mixed_precision_forward": mixed,
            "timing": "wall time between device synchronisations"}


def salame_vs_adjoint(name, iters=8):
    """The beam-loading objective J (current-weighted variance of Ez over the witness slices) of
    the same beams with three witness current profiles: the injected one, the one SALAME makes
    in step 0 (witness.do_salame = 1; SALAME flattens the slice-mean Ez, and removes the witness
    where the target cannot be reached) and the one a few projected gradient-descent steps on the
    adjoint's witness knots reach (backtracking line search; knots kept >= 0, plasma density
    knots fixed). All three are evaluated by the same forward of hpq_adjoint_grad on the initial
    beam positions."""
    import numpy as np
    import hipace2_b200 as hp
    from cases import config
    text = config(name)
    sim = hp.Hipace(text, graphs=True)
    sim.init_data()
    drv0, wit0 = sim.get_beam(0), sim.get_beam(1)
    n_profile = int(_key(text, "adjoint.n_profile_knots"))
    n_density = int(_key(text, "adjoint.n_density_knots"))
    lo, hi = [float(v) for v in _key_all(text, "adjoint.profile_zeta")[:2]]
    ones = np.ones(n_profile + n_density)
    J0 = sim.adjoint(ones, grad=False)
    # SALAME on the same beams (the adjoint keys are left out: the adjoint does not cover SALAME)
    stext = "\n".join(l for l in text.splitlines() if not l.strip().startswith("adjoint.")) + "\nwitness.do_salame = 1\n"
    s = hp.Hipace(stext, graphs=True)
    s.init_data()
    s.set_beam(0, drv0)
    s.set_beam(1, wit0)
    s.step(0)
    ws, log = s.get_beam(1), s.salame_log()
    s.close()
    # SALAME's weights (0 for the particles it removed) on the initial positions
    w_sal = dict(zip(ws["id"].tolist(), ws["w"].tolist()))
    wit_s = dict(wit0)
    wit_s["w"] = np.array([w_sal.get(i, 0.0) for i in wit0["id"].tolist()])
    sim.set_beam(1, wit_s)
    J_sal = sim.adjoint(ones, grad=False)
    sim.set_beam(1, wit0)
    # projected gradient descent on the witness knots
    theta, J, hist, lr = ones.copy(), J0, [J0], None
    for _ in range(iters):
        J, g = sim.adjoint(theta)
        g[n_profile:] = 0.0
        if lr is None:
            lr = 0.25 / max(float(np.abs(g).max()), 1e-300)
        for _try in range(6):
            t = np.maximum(theta - lr * g, 0.0)
            Jt = sim.adjoint(t, grad=False)
            if Jt < J:
                theta, J, lr = t, Jt, lr * 1.5
                break
            lr *= 0.5
        hist.append(J)
    knots_z = np.linspace(lo, hi, n_profile)
    prof = np.where((wit0["z"] >= lo) & (wit0["z"] <= hi), np.interp(wit0["z"], knots_z, theta[:n_profile]), 0.0)
    sim.close()
    return {"workload": name, "objective": "J = S2/S0 - (S1/S0)^2, S_n = sum jz_beam Ez^n over adjoint.objective_zeta",
            "J_injected": J0, "J_salame": J_sal, "J_adjoint_descent": hist,
            "descent_steps": iters, "salame_iterations": int(log.shape[0]),
            "salame_slices": int(np.unique(log[:, 0]).size) if log.size else 0,
            # slices whose witness SALAME removed (W = 0)
            "salame_overloaded_slices": int(np.unique(log[log[:, 2] == 0, 0]).size) if log.size else 0,
            "witness_charge_ratio_salame": float(wit_s["w"].sum() / wit0["w"].sum()),
            "witness_charge_ratio_adjoint": float((wit0["w"] * prof).sum() / wit0["w"].sum())}


def _key(text, key):
    for line in text.splitlines():
        if line.strip().startswith(key + " ") or line.strip().startswith(key + "="):
            return line.split("=", 1)[1].split()[0]
    raise KeyError(key)


def _n_cell(text):
    return [int(v) for v in _key_all(text, "amr.n_cell")]


def _key_all(text, key):
    for line in text.splitlines():
        if line.strip().startswith(key):
            return line.split("=", 1)[1].split()
    raise KeyError(key)


def oracle_run(text, first, n_steps):
    """Whole steps first .. first+n_steps-1 of the FP64 CPU oracle (all slices, beam push
    included) on the beam the oracle draws itself from the deck's seed (the same Philox stream as
    the library's beam injection; no GPU library is loaded). Returns the oracle and the seconds
    spent in the steps."""
    from oracle_lib import Oracle
    o = Oracle(text)
    o.init_beams()
    for s in range(first):
        o.step(s)
    t0 = time.perf_counter()
    for s in range(first, first + n_steps):
        o.step(s)
    return o, time.perf_counter() - t0


def cpu_baseline(text, args):
    """This build's FP64 CPU oracle on a bounded sample of the same workload: its first
    `--cpu-sample-steps` whole steps."""
    n = max(1, args.cpu_sample_steps)
    o, dt = oracle_run(text, 0, n)
    return {"value": o.nz * n / dt, "unit": "slices/s", "cores": o.L.oracle_threads(), "kind": "port",
            "sample": f"steps 0-{n - 1} of {args.config}, every slice of each step with the beam push "
                      "(FP64 oracle, beam drawn by the oracle from the deck's seed)"}


def run_reference(args):
    """Reference arm: the reference's CPU implementation of the path. The reference (AMReX,
    FFTW, MPI) cannot be built on this image, so its FP64 restatement (oracle/, OpenMP, all host
    threads) runs instead, on the same deck: W warm-up steps, then K timed whole steps (every
    slice, beam push included), with the beam the oracle draws from the deck's seed. No GPU
    library is loaded. Under torchrun only rank 0 runs."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from cases import config
    from oracle_lib import Oracle
    text = config(args.config)
    probe = Oracle(text)
    probe.init_beams()
    n_beam0 = int(probe.L.oracle_beam_count(probe.h, 0))
    probe.begin_step(0)  # the plasma of a step is created when the step begins
    n_plasma = int(probe.L.oracle_plasma_count(probe.h, 0))
    grid = (probe.nx, probe.ny, probe.nz)
    del probe
    o, dt = oracle_run(text, args.warmup, args.steps)
    nz = o.nz
    v = nz * args.steps / dt
    threads = o.L.oracle_threads()
    print(json.dumps({
        "impl": "reference", "metric": "slices/s", "value": v, "unit": "slices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded Gaussian driver beam (Philox), lattice plasma",
        "config": workload_config(args, grid, n_plasma, n_beam0, world),
        "cpu_baseline": {"value": v, "unit": "slices/s", "cores": threads, "kind": "port",
                         "sample": f"steps {args.warmup}-{args.warmup + args.steps - 1} of {args.config}, "
                                   "every slice with the beam push; the reference binary is not buildable "
                                   "here (AMReX/FFTW/MPI absent), so its FP64 restatement (oracle/) runs"},
        "e2e": {"value": v, "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
