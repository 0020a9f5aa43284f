#!/usr/bin/env python
"""Benchmark: FP64 Gcell-updates/s of HipFT's flux-transport step on B200.

Workload (default "batched64_1024x2048"): 64 realizations on a 1024 x 2048
(theta x phi) grid whose theta spacing is halved within 15 degrees of each
pole; per-realization diffusion D log-U(100, 1000) km^2/s, meridional flow
v0 U(10, 20) m/s and differential rotation B, C x U(0.9, 1.1) (seed 1);
WENO3-CS(h) + SSPRK(4,3) advection Strang-split with RKG2 super-time-stepped
diffusion (automatic PTL subcycling), assimilation of a synthetic observed
map every 24 model hours (mu^4 weights, mu > 0.1), diagnostics every step.
The configuration is a batch of ragged realizations, so by default every
realization keeps its own schedule (Euler limit, PTL subcycles, RKG2 stage
counts; `--schedule shared` runs the reference's one schedule for all).
A step is one flux-transport time step at the CFL-limited dt of the batch.
Unit of work: one unique grid point of one realization advanced through one
stage (one RKG2 stage or one SSPRK stage).

Timing: W untimed warm-up steps, then K steps between CUDA events on the
library's stream (inputs resident in HBM; each field is 1.07 GB, far above
the 126 MB L2, so no flush is needed), max over ranks.  `e2e` repeats K steps
through the C ABI with the field copied host->device before and
device->host after every step.  Multi-GPU: every rank advances its own batch
of nr realizations (realizations rank*nr .. rank*nr+nr-1 of one parameter
draw) independently -- weak scaling, no data-path collective; `value` is the
cell-stages of all ranks over the slowest rank's time.

At N = 1 the line also carries:
  "batched_vs_plain": realization-steps/s of the ragged batch, of one batch
      on the shared schedule, and of one handle per realization run one
      after another, all at the batch's dt;
  "plain": the same metric for the plain configuration (one realization,
      1024 x 2048, fixed physics, no assimilation), timed step by step with
      an L2 flush before each step (its fields fit in L2);
  "adjoint": gradient / forward cost on the adjoint configuration;
  "cpu_baseline": the CPU oracle's timing build on several realizations.
`--c5` adds the 16-realization 2048 x 4096 forward leg, `--c5-adjoint` the
gradient / forward cost on one of its realizations (flows from files).

`--impl reference` times the CPU oracle (the restatement of the reference's
solver in oracle/, its timing build, all host threads) on a bounded sample
of the same workload: two realizations, one flux-transport step per bench
step.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 Gcell-updates/s"
UNIT = "Gcell-updates/s"
STS_BYTES_PER_CELL = 40  # RKG2 stage k>=2: read Y_{k-1}, Y_{k-2}, u0, dty0; write Y_k
# two-stage kernel per HIPFT_STS_PAIR value (the library's default is 5); the
# timed region of a "launch" is the kernel plus its pole-row launch
STS_KERNELS = {"4": "k_sts_pair_ws+k_pair_poles", "5": "k_sts_pair_ws<rows2>+k_pair_poles",
               "6": "k_sts_pair_ws<rows2, bulk stores>+k_pair_poles"}

WORKLOADS = {
    "batched64_1024x2048": dict(ntm=1024, npm1=2049, nr=64, seed=1),
    "single_1024x2048": dict(ntm=1024, npm1=2049, nr=1, seed=0),
    "batched8_1024x2048": dict(ntm=1024, npm1=2049, nr=8, seed=1),
    "small_128x256": dict(ntm=128, npm1=257, nr=4, seed=1),
}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(0)
        sm, smax, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.tmp.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            try:
                pw.append(float(f[3]))
            except ValueError:
                pass
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.tmp.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w": statistics.median(pw) if pw else None}


def make_inputs(wl: dict, copies: int = 1):
    """Grid, initial map and per-realization parameters of `copies` x nr
    realizations (one batch of nr per GPU when the run is sharded)."""
    from hipft_b200 import synthetic as S
    t = S.refined_theta(wl["ntm"])
    p = S.uniform_phi(wl["npm1"])
    br = S.bipole_map(t, p, wl["seed"])
    prm = S.batched_params(wl["nr"] * copies, wl["seed"])
    return t, p, br, prm


def oracle_sample(t, p, br, prm, dt, indices=(0,)):
    """One flux-transport step of the realizations `indices` on the CPU oracle's
    timing build (liboracle_fast.so: -O3 -march=x86-64-v3 -fopenmp, all host
    threads), at the given dt or, when dt is None, at their own CFL-limited
    dt; returns (cell_updates, seconds)."""
    from oracle import oracle as O
    idx = list(indices)
    q = dict(O.DEFAULTS)
    q.update(n_realizations=len(idx), advance_flow=True, flow_dr_model=1, flow_mf_model=1,
             advance_diffusion=True, strang_splitting=True, flow_num_method=4)
    if dt is None:
        q.update(time_end=1.0e9)
    else:
        q.update(time_end=dt, dt_max=dt)
    raw = {k: v for k, v in q.items()}
    vec = lambda key: [float(prm[key][i]) for i in idx]
    raw.update({
        "diffusion_coef_constants": vec("diffusion_coef_constants"),
        "flow_dr_coef_p0_values": vec("dr_p0"), "flow_dr_coef_p2_values": vec("dr_p2"),
        "flow_dr_coef_p4_values": vec("dr_p4"), "flow_mf_coef_p1_values": vec("mf_p1"),
        "flow_mf_coef_p3_values": vec("mf_p3"), "flow_mf_coef_p5_values": vec("mf_p5"),
    })
    pp = O.process_parameters(raw)
    m = np.ascontiguousarray(np.broadcast_to(br, (len(idx),) + br.shape))
    t0 = time.perf_counter()
    r = O.run(pp, map_pt=m, s1=p, s2=t, want_field=False, hist_cap=16, max_steps=1, fast=True)
    sec = time.perf_counter() - t0
    return r["cell_updates"], sec


def host_threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def run_reference(args, wl, name):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from hipft_b200 import synthetic as S  # noqa: F401  (inputs only)
    t, p, br, prm = make_inputs(wl)
    vals = []
    total = 0.0
    per = 2
    for k in range(args.warmup + args.steps):
        idx = [(per * k + q) % wl["nr"] for q in range(per)]
        cells, sec = oracle_sample(t, p, br, prm, None, indices=idx)
        if k >= args.warmup:
            vals.append(cells / sec / 1e9)
            total += sec
    v = float(np.mean(vals))
    from oracle import oracle as O
    sample = (f"{per} realizations per bench step (cycling through the {wl['nr']}), one Strang flux-transport step "
              f"at their CFL-limited dt on the {wl['ntm']}x{wl['npm1'] - 1} grid; oracle timing build "
              f"{O.FAST_FLAGS}")
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / max(args.steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "grid": [wl["ntm"], wl["npm1"] - 1], "realizations": wl["nr"]},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": host_threads(), "kind": "port", "sample": sample},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def make_handle(H, t, p, br, prm, sl, device, ragged, graph=False):
    """A handle holding realizations `sl` of the workload with its initial map
    and flows loaded; ragged: each realization keeps its own schedule; graph:
    every step runs as one CUDA-graph launch."""
    nrl = len(prm["diffusion_coef_constants"][sl])
    g = H.HipftGPU(t, p, nrl, device=device, advance_flow=True, flow_num_method=4, strang_splitting=True,
                   advance_diffusion=True, diffusion_coef_constants=prm["diffusion_coef_constants"][sl])
    g.load_initial_map(np.broadcast_to(br, (nrl,) + br.shape))
    g.set_flow(dr_model=1, mf_model=1, dr_p0=prm["dr_p0"][sl], dr_p2=prm["dr_p2"][sl], dr_p4=prm["dr_p4"][sl],
               mf_p1=prm["mf_p1"][sl], mf_p3=prm["mf_p3"][sl], mf_p5=prm["mf_p5"][sl])
    g.update_flow()
    if ragged:
        g.set_ragged(True)
    if graph:
        g.set_graph(True)
    return g


def make_step(g, dt, da_times, da_maps, prm, sl, state):
    """One bench step: a flux-transport step, the assimilation when the step
    crosses a 24 h boundary, and the diagnostics."""
    def step():
        g.flux_transport_step(dt)
        state["time"] += dt
        if state["da"] < len(da_times) and state["time"] >= da_times[state["da"]]:
            g.assimilate(da_maps[da_times[state["da"]]], custom_from_mu=True, mu_power=prm["mu_power"][sl],
                         mu_limit=prm["mu_limit"][sl], lat_limit=prm["lat_limit"][sl])
            state["da"] += 1
        g.analysis(state["time"])
    return step


def measure_batched_vs_plain(args, wl, local, t, p, br, prm, dt, da_times, da_maps, ragged_rs_per_s):
    """Realization-steps per second of the same realizations three ways: the
    ragged batch (taken from the timed region), one batch with the shared
    (reference) schedule, and one handle per realization launched one after
    another ("plain per-realization launches"), all at the shared dt."""
    import torch
    import hipft_b200 as H
    stream = torch.cuda.current_stream()
    nr = wl["nr"]
    k = max(2, min(args.steps, 4))
    out = {"unit": "realization-steps/s", "dt_hours": dt, "ragged_batch": ragged_rs_per_s}
    # one batch, shared schedule
    g = make_handle(H, t, p, br, prm, slice(0, nr), local, False)
    g.set_stream(stream.cuda_stream)
    state = {"time": 0.0, "da": 0}
    step = make_step(g, dt, da_times, da_maps, prm, slice(0, nr), state)
    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    out["shared_batch"] = nr * k / (e0.elapsed_time(e1) * 1e-3)
    out["shared_batch_steps"] = k
    g.close()
    # one handle per realization, each with its own schedule
    tot_ms = 0.0
    for i in range(nr):
        gi = make_handle(H, t, p, br, prm, slice(i, i + 1), local, False)
        gi.set_stream(stream.cuda_stream)
        st = {"time": 0.0, "da": 0}
        si = make_step(gi, dt, da_times, da_maps, prm, slice(i, i + 1), st)
        si()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            si()
        b.record(stream)
        torch.cuda.synchronize()
        tot_ms += a.elapsed_time(b)
        gi.close()
    out["per_realization_handles"] = nr * k / (tot_ms * 1e-3)
    out["per_realization_steps"] = k
    out["ragged_over_per_realization"] = ragged_rs_per_s / out["per_realization_handles"]
    out["ragged_over_shared"] = ragged_rs_per_s / out["shared_batch"]
    out["note"] = ("the per-realization handles run one after another, each from the 126 MB L2 (17 MB fields); "
                   "the batches stream 1.07 GB fields from HBM; the shared batch and the per-realization handles run "
                   "host-driven, their faster mode (a one-realization graph-run step is about 8% slower)")
    return out


def run_gpu(args, wl, name):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    from hipft_b200.parallel import reduce_timing, split_realizations

    # weak scaling: every GPU advances its own batch of nr realizations
    # (realizations rank*nr .. rank*nr+nr-1 of one parameter draw); no
    # collective touches the data path
    t, p, br, prm = make_inputs(wl, copies=world)
    first, nrl = split_realizations(wl["nr"] * world, world, rank)
    sl = slice(first, first + nrl)
    ragged = args.schedule == "ragged"
    g = make_handle(H, t, p, br, prm, sl, local, ragged, graph=args.step == "graph")
    stream = torch.cuda.current_stream()
    g.set_stream(stream.cuda_stream)
    dt = g.flow_dtmax()
    ntm, npm = g.ntm, g.npm
    # assimilation maps for every 24 h boundary the run will cross
    n_total = args.warmup + 3 * args.steps + 2
    da_times = [24.0 * k for k in range(1, int(n_total * dt / 24.0) + 2)]
    da_maps = {tt: S.observed_map(t, p, tt, wl["seed"]) for tt in da_times}
    state = {"time": 0.0, "da": 0}
    step = make_step(g, dt, da_times, da_maps, prm, sl, state)

    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    i0 = g.info()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    i1 = g.info()
    cells = float(i1.cell_stage_updates - i0.cell_stage_updates)
    launches = int(i1.kernel_launches - i0.kernel_launches)
    real_steps_per_s = nrl * args.steps / (ms * 1e-3)
    # kernel breakdown in a second pass of the same steps: per-kernel events
    # sit between launches, which the timed pass above keeps free of them
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ip = g.info()
    if args.step == "graph":
        g.set_graph(False)  # per-kernel events need host-driven launches (the same kernels)
    g.set_profiling(True)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(args.steps):
        step()
    p1.record(stream)
    torch.cuda.synchronize()
    ms_prof = p0.elapsed_time(p1)
    sts_n, sts_ms = g.kernel_time(0)
    adv_n, adv_ms = g.kernel_time(1)
    ring_n, ring_ms = g.kernel_time(2)
    oth_n, oth_ms = g.kernel_time(3)
    g.set_profiling(False)
    if args.step == "graph":
        g.set_graph(True)
    ipe = g.info()
    rkg2_stages = int(ipe.rkg2_stages - ip.rkg2_stages)
    rkg2_cell_stages = float(ipe.rkg2_cell_stages - ip.rkg2_cell_stages)
    sched = g.ragged_schedule() if ragged else None

    # end to end through the C ABI with host buffers
    f_host = torch.empty((nrl, npm, ntm), dtype=torch.float64, pin_memory=True).numpy()
    g.get_field(f_host)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    i2 = g.info()
    w0 = time.perf_counter()
    for _ in range(args.steps):
        g.set_field(f_host)
        step()
        g.get_field(f_host)
    w1 = time.perf_counter()
    i3 = g.info()
    e2e_ms = (w1 - w0) * 1e3
    e2e_cells = float(i3.cell_stage_updates - i2.cell_stage_updates)

    if dist:
        ms, cells = reduce_timing(dist, "cuda", ms, cells)
        e2e_ms, e2e_cells = reduce_timing(dist, "cuda", e2e_ms, e2e_cells)
        _, launches = reduce_timing(dist, "cuda", 0.0, float(launches))
        launches = int(launches)

    peak, peak_kind = measured_peak()
    # Algorithmic bytes: 40 B per unique cell per RKG2 stage (read Y_{k-1},
    # Y_{k-2}, u0, dty0; write Y_k), times the cell-stages one launch advances
    # (in a ragged batch a launch covers the realizations with stages left).
    stages_per_launch = rkg2_stages / max(sts_n, 1)
    bytes_per_launch = STS_BYTES_PER_CELL * rkg2_cell_stages / max(sts_n, 1)
    sts_avg_ms = sts_ms / max(sts_n, 1)
    achieved = bytes_per_launch / (sts_avg_ms * 1e-3) / 1e9 if sts_n else None
    traffic, traffic_src = None, None
    sts_kernel = STS_KERNELS.get(os.environ.get("HIPFT_STS_PAIR", "5"), STS_KERNELS["5"]) if stages_per_launch > 1.5 \
        else "k_sts_stage_v3"
    tpath = os.path.join(ROOT, "profiles", "sts_stage_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as fh:
            tj = json.load(fh)
        if abs(tj.get("stages_per_launch", 1) - stages_per_launch) < 1e-9 and tj.get("kernel") == sts_kernel:
            traffic = tj["dram_bytes_per_cell"] * ntm * (npm - 2) * nrl
            traffic_src = tj["source"]
    out = {
        "metric": METRIC, "value": cells / (ms * 1e-3) / 1e9, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": name, "grid": [ntm, npm - 2], "realizations": wl["nr"] * world,
                   "realizations_per_gpu": nrl, "dt_hours": dt,
                   "parallelism": f"replicas: {world} GPU(s), {nrl} realizations each",
                   "schedule": ("ragged: each realization its own Euler limit, PTL subcycles and RKG2 stage "
                                "counts" if ragged else "shared (the reference's MIN/MAX schedule)"),
                   "method": "WENO3+SSPRK(4,3) Strang-split with RKG2 (PTL subcycles), DA every 24 h",
                   "step": ("one CUDA-graph launch per split step (PTL subcycles, stage counts and substeps "
                            "decided on the device)" if args.step == "graph" else "host-driven launches"),
                   "l2": "inputs larger than L2 (%.2f GB per field), no flush" % (ntm * npm * nrl * 8 / 1e9)},
        "roofline": {"bound": "hbm",
                     "kernel": sts_kernel, "kernel_role": ("two fused RKG2 stages per launch"
                                                           if stages_per_launch > 1.5 else "one fused RKG2 stage"),
                     "stages_per_launch": stages_per_launch, "traffic_source": traffic_src,
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "launches": sts_n, "avg_launch_ms": sts_avg_ms,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "share_of_step": sts_ms / ms_prof if ms_prof > 0 else None,
                     "timing": "per-kernel CUDA events in a second pass of the same steps",
                     "kernels_over_step": ((sts_ms + adv_ms + ring_ms + oth_ms) / ms_prof) if ms_prof > 0 else None,
                     "other_kernels_ms": {"advection_stage": adv_ms, "ring_sums": ring_ms, "other": oth_ms},
                     "other_kernels_launches": {"advection_stage": adv_n, "ring_sums": ring_n, "other": oth_n}},
        "e2e": {"value": e2e_cells / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
                "h2d_bytes_per_step": ntm * npm * nrl * 8, "d2h_bytes_per_step": ntm * npm * nrl * 8},
        "gpu_launches": launches,
        "clocks": clk,
        "realization_steps_per_s": real_steps_per_s,
    }
    out["config"]["kernels"] = g.describe()
    if sched is not None:
        out["config"]["rkg2_stages_per_realization"] = [int(x) for x in sched["sts_s"]]
        out["config"]["subcycles_per_realization"] = [int(x) for x in sched["subcycles"]]
    if rank == 0 and world == 1 and not args.no_plain:
        out["batched_vs_plain"] = measure_batched_vs_plain(args, wl, local, t, p, br, prm, dt, da_times, da_maps,
                                                           real_steps_per_s)
    if rank == 0 and world == 1 and not args.no_plain:
        out["plain"] = measure_plain(args, local)
    if rank == 0 and world == 1 and not args.no_adjoint:
        out["adjoint"] = measure_adjoint(args, local, days=args.adjoint_days)
    if rank == 0 and world == 1 and args.c5:
        out["c5"] = measure_c5(args, local)
    if rank == 0 and world == 1 and args.c5_adjoint:
        out["c5_adjoint"] = measure_c5_adjoint(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        idx = [0, 1, 2, 3]
        cells_c, sec_c = oracle_sample(t, p, br, prm, dt, indices=idx)
        out["cpu_baseline"] = {"value": cells_c / sec_c / 1e9, "unit": UNIT, "cores": host_threads(),
                               "kind": "port",
                               "sample": f"CPU oracle timing build ({O.FAST_FLAGS}), realizations {idx} of the batch, "
                                         f"one Strang flux-transport step of dt={dt:.4f} h with their shared schedule "
                                         f"({sec_c:.1f} s)"}
    if rank == 0:
        print(json.dumps(out))
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def measure_plain(args, local: int):
    """The plain configuration beside the batched one: one realization on the
    same 1024 x 2048 refined grid with fixed physics (D 300 km^2/s, v0 15 m/s,
    B -2.40, C -1.80 deg/day), no assimilation.  Its fields (17 MB) fit in L2,
    so a 256 MB buffer is written between timed steps and each step is timed
    alone; e2e adds the host copies of the field."""
    import torch
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    wl = WORKLOADS["single_1024x2048"]
    t = S.refined_theta(wl["ntm"])
    p = S.uniform_phi(wl["npm1"])
    br = S.bipole_map(t, p, wl["seed"])
    prm = S.plain_params()
    g = H.HipftGPU(t, p, 1, device=local, advance_flow=True, flow_num_method=4, strang_splitting=True,
                   advance_diffusion=True, diffusion_coef_constants=prm["diffusion_coef_constants"])
    stream = torch.cuda.current_stream()
    g.set_stream(stream.cuda_stream)
    g.load_initial_map(br[None])
    g.set_flow(dr_model=1, mf_model=1, dr_p0=prm["dr_p0"], dr_p2=prm["dr_p2"], dr_p4=prm["dr_p4"],
               mf_p1=prm["mf_p1"], mf_p3=prm["mf_p3"], mf_p5=prm["mf_p5"])
    g.update_flow()
    dt = g.flow_dtmax()
    ntm, npm = g.ntm, g.npm
    state = {"time": 0.0}

    def step():
        g.flux_transport_step(dt)
        state["time"] += dt
        g.analysis(state["time"])

    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device=f"cuda:{local}")  # 256 MB > L2
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def timed(profile: bool):
        info0 = g.info()
        g.set_profiling(profile)
        tot = 0.0
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return info0, g.info(), tot

    i0, i1, ms = timed(False)
    ip, ip1, ms_prof = timed(True)
    sts_n, sts_ms = g.kernel_time(0)
    g.set_profiling(False)
    cells = float(i1.cell_stage_updates - i0.cell_stage_updates)
    rkg2 = int(ip1.rkg2_stages - ip.rkg2_stages)
    f_host = torch.empty((1, npm, ntm), dtype=torch.float64, pin_memory=True).numpy()
    g.get_field(f_host)
    torch.cuda.synchronize()
    i2 = g.info()
    w = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        g.set_field(f_host)
        step()
        g.get_field(f_host)
        w += time.perf_counter() - w0
    i3 = g.info()
    peak, peak_kind = measured_peak()
    spl = rkg2 / max(sts_n, 1)
    avg = sts_ms / max(sts_n, 1)
    achieved = STS_BYTES_PER_CELL * ntm * (npm - 2) * spl / (avg * 1e-3) / 1e9 if sts_n else None
    out = {"workload": "single_1024x2048", "grid": [ntm, npm - 2], "realizations": 1, "dt_hours": dt,
           "value": cells / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms / args.steps, "steps": args.steps,
           "l2": "256 MB buffer written before every timed step, each step timed alone (fields fit in L2)",
           "e2e": {"value": float(i3.cell_stage_updates - i2.cell_stage_updates) / w / 1e9, "unit": UNIT,
                   "h2d_bytes_per_step": ntm * npm * 8, "d2h_bytes_per_step": ntm * npm * 8},
           "roofline": {"kernel": STS_KERNELS.get(os.environ.get("HIPFT_STS_PAIR", "5"), STS_KERNELS["5"]),
                        "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                        "avg_launch_ms": avg, "launches": sts_n,
                        "share_of_step": sts_ms / ms_prof if ms_prof > 0 else None,
                        "note": "L2-resident after the first stages of a step; a fraction of the HBM copy "
                                "bandwidth is not a DRAM measurement here"},
           "gpu_launches": int(i1.kernel_launches - i0.kernel_launches)}
    g.close()
    del flush
    return out


def measure_adjoint(args, local: int, days: float = 27.27, checkpoint_every: int = 64):
    """Gradient / forward cost of the misfit adjoint on the adjoint
    configuration: 512 x 1024 uniform grid, one realization, the plain
    configuration's physics (D 300 km^2/s, v0 15 m/s, B -2.40, C -1.80
    deg/day) with PTL subcycling, `days` of model time at the CFL-limited dt,
    a checkpoint every `checkpoint_every` steps (so the segment recompute is
    inside the gradient's time).  Wall time of MisfitAdjoint.run (forward with
    checkpoints, misfit, recompute, replay, reverse) over the same steps
    through the library's forward alone (field copied in and out).  The
    target map is the same run with D x 1.2 and v0 + 3 m/s."""
    import torch
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    from hipft_b200.adjoint import MisfitAdjoint
    ntm, npm1 = 512, 1025
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    br = S.bipole_map(t, p, 0)
    prm = S.plain_params()
    flow = {"p0": prm["dr_p0"], "p2": prm["dr_p2"], "p4": prm["dr_p4"], "p1": prm["mf_p1"], "p3": prm["mf_p3"],
            "p5": prm["mf_p5"]}

    def handle(D, fl):
        g = H.HipftGPU(t, p, 1, device=local, advance_flow=True, flow_num_method=4, strang_splitting=True,
                       advance_diffusion=True, diffusion_coef_constants=D)
        g.set_flow(dr_model=1, mf_model=1, dr_p0=fl["p0"], dr_p2=fl["p2"], dr_p4=fl["p4"], mf_p1=fl["p1"],
                   mf_p3=fl["p3"], mf_p5=fl["p5"])
        return g

    D = prm["diffusion_coef_constants"]
    g = handle(D, flow)
    g.load_initial_map(br[None])
    f0 = g.get_field()
    g.update_flow()
    dt = g.flow_dtmax()
    tend = 24.0 * days
    dts, time_ = [], 0.0
    while time_ < tend:
        d = min(dt, tend - time_)
        dts.append(d)
        time_ += d

    def forward(gg, f):
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        gg.set_field(f)
        gg.update_flow()
        for d in dts:
            gg.flux_transport_step(d)
        out = gg.get_field()
        torch.cuda.synchronize()
        return out, time.perf_counter() - w0

    fl_t = dict(flow, p1=flow["p1"] + 6.0, p3=flow["p3"] - 6.0)
    gt = handle(D * 1.2, fl_t)
    target, _ = forward(gt, f0)
    gt.close()
    forward(g, f0)
    import gc
    gc.collect()
    gc.disable()
    fwd_runs = [forward(g, f0)[1] for _ in range(5)]
    gc.enable()
    A = MisfitAdjoint(g, D, flow, checkpoint_every=checkpoint_every)
    A.run(f0, target, dts)  # warm-up: tuner, tape allocation (kept by the handle)
    grad_runs, phases = [], []
    import gc
    for _ in range(5):
        gc.collect()
        gc.disable()  # no collector pauses inside a timed run
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        loss, grads = A.run(f0, target, dts)
        torch.cuda.synchronize()
        grad_runs.append(time.perf_counter() - w0)
        gc.enable()
        phases.append({"forward_s": A.timing.get("forward_s"), "forward_parts": A.timing.get("forward_parts"),
                       "reverse_s": A.timing.get("reverse_s"),
                       "segments": A.timing.get("segments")})
    fwd_s, grad_s = statistics.median(fwd_runs), statistics.median(grad_runs)
    tape = ctypes.c_int64(0)
    g.L.hipft_adj_tape_fields(g.h, ctypes.byref(tape))
    if args.adjoint_kernels:
        # per-kernel device times of one more gradient, through CUPTI (torch.profiler), to stderr
        from torch.profiler import profile, ProfilerActivity
        with profile(activities=[ProfilerActivity.CUDA]) as pr:
            A.run(f0, target, dts)
            torch.cuda.synchronize()
        rows = sorted([(e.key, e.count, e.device_time_total) for e in pr.key_averages() if e.device_time_total > 0],
                      key=lambda r: -r[2])
        tot = sum(r[2] for r in rows)
        print(f"adjoint gradient: device total {tot / 1e3:.1f} ms (kernels may overlap)", file=sys.stderr)
        for key, cnt, tt in rows[:12]:
            print(f"  {tt / 1e3:9.2f} ms {100 * tt / tot:5.1f}% {cnt:7d}x {tt / max(cnt, 1):8.2f} us  {key[:80]}",
                  file=sys.stderr)
    A.release()
    g.close()
    return {"workload": "adjoint_512x1024", "grid": [ntm, npm1 - 1], "realizations": 1, "steps": len(dts),
            "model_days": days, "dt_hours": dt, "subcycling": "PTL (automatic)",
            "checkpoint_every": checkpoint_every, "segments": -(-len(dts) // checkpoint_every),
            "forward_ms": fwd_s * 1e3, "gradient_ms": grad_s * 1e3, "gradient_over_forward": grad_s / fwd_s,
            "runs": "median of 5 timed runs each", "forward_runs_ms": [x * 1e3 for x in fwd_runs],
            "gradient_runs_ms": [x * 1e3 for x in grad_runs], "gradient_phases": phases,
            "loss": loss, "grad_D": float(grads["D"][0]), "grad_f0_norm": float(np.linalg.norm(grads["f0"])),
            "tape_fields_peak": int(tape.value),
            "tape_gb_peak": int(tape.value) * ntm * (npm1 + 1) * 8 / 1e9,
            "note": "wall times with host copies of the field; the gradient covers the forward with its "
                    "checkpoints and the taped last segment, the taped recompute of the other segments from "
                    "their checkpoints, and the reverse kernels"}


def measure_c5(args, local: int, steps: int = 2):
    """The large configuration's forward leg: 16 realizations (seed 2, the
    64-realization configuration's parameter ranges) on 2048 x 4096 with theta
    refined near the poles, the random divergent supergranular flow of day 0
    (30 Mm, 300 m/s rms; shared by the realizations, as HipFT's flow files are)
    under each realization's analytic differential rotation and meridional
    flow, ragged schedule, a few steps at the CFL-limited dt."""
    import torch
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    ntm, npm1, nr, seed = 2048, 4097, 16, 2
    t = S.refined_theta(ntm)
    p = S.uniform_phi(npm1)
    br = S.bipole_map(t, p, seed)
    prm = S.batched_params(nr, seed)
    w0 = time.perf_counter()
    vt, vp = S.supergranular_flow(t, p, seed, day=0, coarse=(256, 513))
    gen_s = time.perf_counter() - w0
    g = H.HipftGPU(t, p, nr, device=local, advance_flow=True, flow_num_method=4, strang_splitting=True,
                   advance_diffusion=True, diffusion_coef_constants=prm["diffusion_coef_constants"])
    stream = torch.cuda.current_stream()
    g.set_stream(stream.cuda_stream)
    g.load_initial_map(np.broadcast_to(br, (nr,) + br.shape))
    g.set_flow_from_files(vt, vp, at_load=True)
    g.set_flow(dr_model=1, mf_model=1, dr_p0=prm["dr_p0"], dr_p2=prm["dr_p2"], dr_p4=prm["dr_p4"],
               mf_p1=prm["mf_p1"], mf_p3=prm["mf_p3"], mf_p5=prm["mf_p5"])
    g.update_flow()
    g.set_ragged(True)
    dt = g.flow_dtmax()
    g.flux_transport_step(dt)
    torch.cuda.synchronize()
    i0 = g.info()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        g.update_flow()
        g.flux_transport_step(dt)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    i1 = g.info()
    sched = g.ragged_schedule()
    out = {"workload": "batched16_2048x4096", "grid": [ntm, npm1 - 1], "realizations": nr, "steps": steps,
           "dt_hours": dt, "ms_per_step": ms / steps,
           "value": float(i1.cell_stage_updates - i0.cell_stage_updates) / (ms * 1e-3) / 1e9, "unit": UNIT,
           "realization_steps_per_s": nr * steps / (ms * 1e-3),
           "rkg2_stages_per_realization": [int(x) for x in sched["sts_s"]],
           "device_bytes": int(i1.device_bytes), "flow_generation_s": gen_s,
           "note": "flows from the supergranular generator through hipft_gpu_set_flow_from_files, rebuilt at "
                   "every update_flow as HipFT does while flows come from files"}
    g.close()
    return out


def measure_c5_adjoint(args, local: int, steps: int = 6, checkpoint_every: int = 2, runs: int = 3):
    """Gradient / forward cost on one realization of the 16-realization
    2048 x 4096 configuration (its realization 0: D, differential rotation and
    meridional flow of seed 2, the supergranular flow of day 0 from files),
    plain schedule with PTL subcycling, `steps` steps at the CFL-limited dt,
    a checkpoint every `checkpoint_every` steps.  The batch's gradient runs
    realization by realization: a stage-checkpointed step tape of one
    realization is about 2 + 2 sqrt(2 s) fields of 67 MB.  Target: the same
    run with D x 1.2."""
    import torch
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    from hipft_b200.adjoint import MisfitAdjoint
    ntm, npm1, seed = 2048, 4097, 2
    t = S.refined_theta(ntm)
    p = S.uniform_phi(npm1)
    br = S.bipole_map(t, p, seed)
    prm = S.batched_params(16, seed)
    flow = {"p0": prm["dr_p0"][:1], "p2": prm["dr_p2"][:1], "p4": prm["dr_p4"][:1], "p1": prm["mf_p1"][:1],
            "p3": prm["mf_p3"][:1], "p5": prm["mf_p5"][:1]}
    vt, vp = S.supergranular_flow(t, p, seed, day=0, coarse=(256, 513))
    D = prm["diffusion_coef_constants"][:1]

    def handle(Dv):
        g = H.HipftGPU(t, p, 1, device=local, advance_flow=True, flow_num_method=4, strang_splitting=True,
                       advance_diffusion=True, diffusion_coef_constants=Dv)
        g.set_flow_from_files(vt, vp, at_load=True)
        g.set_flow(dr_model=1, mf_model=1, dr_p0=flow["p0"], dr_p2=flow["p2"], dr_p4=flow["p4"],
                   mf_p1=flow["p1"], mf_p3=flow["p3"], mf_p5=flow["p5"])
        return g

    g = handle(D)
    g.load_initial_map(br[None])
    f0 = g.get_field()
    g.update_flow()
    dts = [g.flow_dtmax()] * steps

    def forward(gg, f):
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        gg.set_field(f)
        gg.update_flow()
        for d in dts:
            gg.flux_transport_step(d)
        out = gg.get_field()
        torch.cuda.synchronize()
        return out, time.perf_counter() - w0

    gt = handle(D * 1.2)
    target, _ = forward(gt, f0)
    gt.close()
    forward(g, f0)
    fwd_runs = [forward(g, f0)[1] for _ in range(runs)]
    A = MisfitAdjoint(g, D, flow, checkpoint_every=checkpoint_every)
    A.run(f0, target, dts)  # warm-up: tuner, tape allocation
    grad_runs = []
    for _ in range(runs):
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        A.run(f0, target, dts)
        torch.cuda.synchronize()
        grad_runs.append(time.perf_counter() - w0)
    tape = A._tape_fields()
    info = g.info()
    fbytes = A._fbytes
    A.release()
    g.close()
    fw, gr = statistics.median(fwd_runs), statistics.median(grad_runs)
    return {"workload": "adjoint_c5_realization0_2048x4096", "grid": [ntm, npm1 - 1], "realizations": 1,
            "steps": steps, "dt_hours": dts[0], "checkpoint_every": checkpoint_every,
            "flows": "supergranular flow of day 0 from files + analytic differential rotation and meridional flow",
            "forward_ms": fw * 1e3, "gradient_ms": gr * 1e3, "gradient_over_forward": gr / fw,
            "runs": f"median of {runs}", "tape_fields": int(tape), "field_bytes": int(fbytes),
            "tape_gb": tape * fbytes / 1e9, "handle_device_gb": info.device_bytes / 1e9}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hipft", choices=["hipft", "reference"])
    ap.add_argument("--workload", default="batched64_1024x2048", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain (one realization) leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the gradient / forward cost leg")
    ap.add_argument("--c5", action="store_true", help="add the 16-realization 2048 x 4096 forward leg")
    ap.add_argument("--c5-adjoint", action="store_true",
                    help="add the gradient / forward cost on one realization of the 2048 x 4096 configuration")
    ap.add_argument("--adjoint-days", type=float, default=27.27,
                    help="model days of the adjoint leg (27.27: the adjoint configuration)")
    ap.add_argument("--adjoint-kernels", action="store_true",
                    help="print the adjoint gradient's per-kernel device times (CUPTI) to stderr")
    ap.add_argument("--step", default="graph", choices=["graph", "host"],
                    help="graph: each split step is one CUDA-graph launch; host: host-driven launches")
    ap.add_argument("--schedule", default="ragged", choices=["ragged", "shared"],
                    help="ragged: every realization its own schedule (default); shared: the reference's")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, wl, args.workload)
    return run_gpu(args, wl, args.workload)


if __name__ == "__main__":
    sys.exit(main())
