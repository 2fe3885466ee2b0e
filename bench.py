"""Benchmark of the forward dynamic-rupture time step on B200.

Workload (default): the 600x300x240 curvilinear case -- Gaussian-hill
topography, four-layer medium with a 3% smoothed perturbation, vertical
split-node fault of 400x180 nodes with linear slip-weakening friction,
20-layer CFS-PML, traction-image free surface, 32 stations -- built from
seeded synthetic inputs (gpu-cgfd3d-dynamic_b200/inputs.py: hills_layered).
A step is one full time step (4 RK stages) of the whole domain.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  value = grid-point updates per second over
the K timed steps (CUDA events on the solver's stream, max over ranks);
inputs (four wavefield levels of 9 components: 6.6 GB per GPU on the
600x300x240 case, 42 GB on 1200x600x400) exceed the 126 MB L2, so no
flush is needed between steps.  --gpus N runs N independent replicas (one
per GPU): the forward path does not shard.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu-cgfd3d-dynamic_b200")
sys.path.insert(0, PKG)

BYTES_PER_POINT_STEP = 768          # algorithmic HBM traffic of one point and step (FP32)
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hills", choices=["hills", "hills_medium", "tpv", "large"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the extra measurement of the 1200x600x400 case in the default run")
    ap.add_argument("--ensemble", type=int, default=0, metavar="N",
                    help="batched form: N seeded scenarios of uneven size advanced as one ensemble, against a "
                         "loop of the plain solver over the same scenarios; prints scenarios/hour")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="steps of the end-to-end run (default: the workload's own run length, e.g. the 3000 "
                         "steps of the 600x300x240 case, so that the one-time upload is amortised as in a real run)")
    return ap.parse_args()


# the length of a whole run of each workload (time steps): the end-to-end
# figure covers one such run, the one-time upload included
RUN_STEPS = {"hills": 3000, "hills_medium": 3000, "tpv": 600, "large": 4000}


def make_problem(workload):
    import inputs
    if workload == "tpv":
        return inputs.tpv_planar(), "tpv_planar 160x100x80 (x strike, y normal, z depth), h=200 m, homogeneous, planar fault"
    if workload == "large":
        return (inputs.hills_layered(ni=600, nj=1200, nk=400, h=50.0, pml=20, fault_len=800, fault_depth=360,
                                     nuc_half=30, dip=25.0, vk_stress=True, nt=4000),
                "hills_layered 1200x600x400 (x strike, y normal, z depth), h=50 m, 8 hills, 4 layers +3%, "
                "25-degree dipping fault 800x360 nodes, von Karman shear stress, 20-layer CFS-PML, 32 stations")
    if workload == "hills_medium":
        # the same construction at 300x200x160 (2 GB on the device): the case
        # the ncu captures of the kernels run on
        return (inputs.hills_layered(ni=200, nj=300, nk=160, pml=20, nsta=8, fault_len=200, fault_depth=120,
                                     margin=20, nhills=4),
                "hills_layered 300x200x160 (x strike, y normal, z depth), h=100 m, 4 hills, 200x120-node fault")
    return inputs.hills_layered(), ("hills_layered 600x300x240 (x strike, y normal, z depth), h=100 m, "
                                    "8 Gaussian hills, 4-layer medium +3% perturbation, 400x180-node fault, "
                                    "20-layer CFS-PML, free surface, 32 stations")


def dist_init():
    import replicas
    return replicas.init("nccl")


def barrier(ws):
    import replicas
    replicas.barrier(ws)


def allmax(ws, x):
    import replicas
    return replicas.allmax(ws, x, "cuda")


class ClockSampler:
    """nvidia-smi samples (every 200 ms) of SM clock, power and throttle
    reasons; stop() keeps the samples taken inside the timed region."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def wait_first_sample(self, timeout_s=10.0):
        """Block until nvidia-smi has written a sample (it takes up to a
        second to start), so that the timed region is covered."""
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < timeout_s:
            if os.path.getsize(self.f.name) > 0:
                return True
            time.sleep(0.05)
        return False

    @staticmethod
    def _stamp(t):
        import datetime
        try:
            return datetime.datetime.strptime(t.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def stop(self, t_start=None, t_end=None):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 10]
        os.unlink(self.f.name)
        if t_start is not None:
            inside = [r for r in rows if (self._stamp(r[0]) or 0) >= t_start - 0.2 and
                      (self._stamp(r[0]) or 0) <= t_end + 0.2]
            rows = inside or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        load = [r for r in rows if r[5].strip().isdigit() and int(r[5]) >= 50] or rows
        sm = [float(r[2]) for r in load if r[2].strip().replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].strip().replace(".", "").isdigit()]
        pw = [float(r[4]) for r in load if r[4].strip().replace(".", "").isdigit()]
        reasons = sorted({n for r in load for n, v in zip(names, r[7:11]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w": statistics.median(pw) if pw else None,
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(load)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(points):
    """DRAM bytes (read + write) of one interior-kernel launch, from the
    committed ncu figures (captured on the medium case, averaged over the RK
    stage kinds and scaled by the points the launch updates)."""
    try:
        with open(os.path.join(ROOT, "profiles", "interior_traffic.json")) as f:
            d = json.load(f)
        return d["dram_bytes_per_point"] * points
    except Exception:
        return None


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def oracle_rate(prob, steps, warmup, budget_s=150.0):
    """CPU oracle on the same problem; returns (Gpt/s, cores, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import OracleSolver
    th = cpu_threads()
    o = OracleSolver(prob, threads=th)
    for _ in range(min(warmup, 1)):
        o.run(1)
    t = time.perf_counter()
    o.run(1)
    one = time.perf_counter() - t
    n = 1
    more = max(0, min(steps, int(budget_s / max(one, 1e-3))) - 1)
    if more:
        t = time.perf_counter()
        o.run(more)
        one = (one + (time.perf_counter() - t)) / (1 + more)
        n += more
    o.close()
    return prob.points / one / 1e9, th, f"{n} full time step(s) of the same problem after set-up, {th} OpenMP threads"


def large_case(peak, setup_free=None, warmup=3, steps=10):
    """The 1200x600x400 case (288 M points, 25-degree dipping fault, von
    Karman stress; about 66 GB on the device) measured after the main
    workload with the same device timing: device Gpt-updates/s, the
    interior kernel's and the whole step's fraction of the HBM peak."""
    import torch
    import cgfd
    if setup_free is not None:
        setup_free.close()
    cgfd.load_library().cgfd_release_cached_memory()
    prob, desc = make_problem("large")
    t0 = time.perf_counter()
    s = cgfd.Solver(prob)
    t_up = time.perf_counter() - t0
    s.run(warmup)
    s.set_timing(True)
    torch.cuda.synchronize()
    s.run(steps)
    run_ms, _, _ = s.last_timing()
    int_ms, int_n, int_pts = s.kernel_timing(1)
    s.close()
    del s
    cgfd.load_library().cgfd_release_cached_memory()
    value = prob.points * steps / (run_ms / 1e3) / 1e9
    achieved = int_pts * BYTES_PER_POINT_STEP / 4 / (int_ms / int_n / 1e3) / 1e9 if int_n else 0.0
    return {"workload": desc, "grid": [prob.nj, prob.ni, prob.nk], "points": prob.points, "steps": steps,
            "warmup": warmup, "value": value, "unit": "Gpt/s", "ms_per_step": run_ms / steps,
            "interior_frac": achieved / peak, "step_frac": value * BYTES_PER_POINT_STEP / peak,
            "setup_and_upload_s": round(t_up, 1),
            "note": "device time of the same kind as value; l2: inputs larger than L2 (42 GB of wavefield levels)"}


def ensemble_main(args):
    """Scenarios per hour of 1500-step runs, from --steps timed steps of
    every scenario: the ensemble (one graph launch per step, a branch per
    scenario) against looping cgfd_run over the same solvers.  Under
    torchrun the scenarios are partitioned across the ranks by cost (points
    x steps, shard.partition), each rank running its share as one ensemble
    on its own GPU; the job's time is the slowest rank's."""
    import torch
    import cgfd
    import inputs
    import shard
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    probs = inputs.ensemble_scenarios(args.ensemble, nt=args.warmup + 2 * args.steps + 16)
    parts = shard.partition([shard.scenario_cost(p, 1500) for p in probs], ws)
    mine = [probs[q] for q in parts[rank]]
    solvers = [cgfd.Solver(p) for p in mine]
    pts = sum(p.points for p in probs)
    for s in solvers:                              # warm-up: graphs of every operator pair
        s.run(max(args.warmup, 8))
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    for s in solvers:
        s.run(args.steps)
    torch.cuda.synchronize()
    t_loop = allmax(ws, time.perf_counter() - t0)
    ens = cgfd.Ensemble(solvers) if solvers else None
    if ens:
        ens.run(8)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.wait_first_sample()
    barrier(ws)
    t_start = time.time()
    t0 = time.perf_counter()
    if ens:
        ens.run(args.steps)
    torch.cuda.synchronize()
    t_ens = allmax(ws, time.perf_counter() - t0)
    clocks = clk.stop(t_start, time.time())
    full = 1500
    rate = lambda t: len(probs) * 3600.0 / (t * full / args.steps)
    line = {"metric": "ensemble scenarios/hour", "value": rate(t_ens), "unit": "scenarios/h",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "strong",
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(probs)} seeded scenarios (inputs.ensemble_scenarios): grids "
                                   "64-160 x 96-256 x 64-128, h 100-200 m, von Karman shear stress, random "
                                   "nucleation, mu_s 0.6-0.7, Dc 0.2-0.5 m, half with hill topography; "
                                   f"{full}-step runs, rate from {args.steps} timed steps of every scenario",
                       "points": pts,
                       "parallelism": f"scenarios partitioned by cost over {ws} GPUs" if ws > 1 else "single GPU"},
            "loop": {"value": rate(t_loop), "unit": "scenarios/h",
                     "note": "cgfd_run over the same solvers one after another"},
            "speedup_vs_loop": t_loop / t_ens,
            "gpt_per_s": pts * args.steps / t_ens / 1e9, "clocks": clocks}
    if ens:
        ens.close()
    barrier(ws)
    if rank == 0:
        print(json.dumps(line), flush=True)
    import replicas
    replicas.finish(ws)


def main():
    args = parse()
    if args.ensemble:
        return ensemble_main(args)
    ws, rank, local = dist_init()
    prob, desc = make_problem(args.workload)
    metric, unit = "Gpt-updates/s", "Gpt/s"
    config = {"workload": desc, "grid": [prob.nj, prob.ni, prob.nk], "points": prob.points,
              "dt": prob.dt, "dynamic_method": prob.dynamic_method,
              "l2": f"inputs larger than L2 ({4 * 9 * 4 * (prob.ni + 6) * (prob.nj + 6) * (prob.nk + 6) / 1e9:.1f} GB "
                    "of wavefield levels), no flush",
              "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"}

    if args.impl == "reference":
        if rank != 0:
            return
        v, th, sample = oracle_rate(prob, args.steps, args.warmup)
        line = {"impl": "reference", "metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": unit, "cores": th, "kind": "port", "sample": sample},
                "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference has no CPU implementation; the CPU oracle restating its "
                        "algorithm stands in for it"}
        print(json.dumps(line), flush=True)
        return

    import torch
    import cgfd
    torch.cuda.set_device(local)
    setup = cgfd.Setup(prob)
    s = cgfd.Solver(prob, setup=setup)
    clk = ClockSampler(local)
    s.run(args.warmup)
    s.set_timing(True)
    clk.wait_first_sample()
    barrier(ws)
    torch.cuda.synchronize()
    t_start = time.time()
    s.run(args.steps)
    torch.cuda.synchronize()
    t_end = time.time()
    clocks = clk.stop(t_start, t_end)
    barrier(ws)
    run_ms, vol_ms, vol_n = s.last_timing()
    int_ms, int_n, int_pts = s.kernel_timing(1)
    _, _, vol_pts = s.kernel_timing(0)
    launches = s.last_launches()
    run_ms_max = allmax(ws, run_ms)
    vol_ms_max = allmax(ws, vol_ms)
    int_ms_max = allmax(ws, int_ms)
    import replicas
    value = replicas.aggregate_rate(prob.points, args.steps, ws, run_ms_max / 1e3) / 1e9
    peak, peak_kind = peaks()
    # dominant kernel: the interior-box volume kernel; one launch is one RK
    # stage of int_pts points at 768 / 4 = 192 algorithmic bytes each
    bytes_per_launch = int_pts * BYTES_PER_POINT_STEP / 4
    achieved = bytes_per_launch / (int_ms_max / int_n / 1e3) / 1e9 if int_n else 0.0
    stage_bytes = vol_pts * BYTES_PER_POINT_STEP / 4
    stage_achieved = stage_bytes / (vol_ms_max / vol_n / 1e3) / 1e9
    tr = traffic_per_launch(int_pts)
    s.close()

    # end to end through the C ABI with host buffers: upload of the prepared
    # problem, then the run with the 11 fault fields read back before every
    # step (the reference's per-step fault output, io_time_skip = 1) into
    # page-locked host memory by cgfd_run_fault_output, in calls of CHUNK
    # steps, stations at the end -- the span of the reference's own timed
    # region (drv_rk_curv_col_allstep)
    ke = args.e2e_steps or RUN_STEPS.get(args.workload, max(args.steps, 100))
    chunk = 20
    nbytes_f = 11 * prob.nk * prob.nj * 4 * prob.num_faults
    pinned = torch.empty(chunk * nbytes_f // 4, dtype=torch.float32, pin_memory=True)
    clk2 = ClockSampler(local)
    clk2.wait_first_sample()
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t0_wall = time.time()
    s2 = cgfd.Solver(prob, setup=setup)
    t_up = time.perf_counter() - t0
    done = 0
    while done < ke:
        n = min(chunk, ke - done)
        s2.run_fault_output(n, 1, out_ptr=pinned.data_ptr(), max_records=chunk)
        done += n
    seis = s2.stations()
    torch.cuda.synchronize()
    e2e_s = allmax(ws, time.perf_counter() - t0)
    e2e_clocks = clk2.stop(t0_wall, time.time())
    s2.close()
    up = setup.upload_bytes
    e2e = {"value": prob.points * ke * ws / e2e_s / 1e9, "unit": unit,
           "h2d_bytes_per_step": int(up / ke), "d2h_bytes_per_step": int(nbytes_f + seis.nbytes / ke),
           "steps": ke, "upload_s": round(t_up, 4), "steps_s": round(e2e_s - t_up, 4),
           "ms_per_step": round((e2e_s - t_up) / ke * 1e3, 3), "clocks": e2e_clocks,
           "note": "the workload's whole run: upload of the prepared problem amortised over its steps; "
                   "host set-up excluded; the fault fields of every step copied to page-locked host memory by "
                   f"cgfd_run_fault_output in calls of {chunk} steps; a run this long reaches the GPU's power "
                   "limit (clocks: SM clock and power sampled over this run), so its ms_per_step is the "
                   "sustained one, the device-timed value above the burst one"}

    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "roofline": {"bound": "hbm", "kernel": "k_volume<INTERIOR> (fused RK stage of the interior box)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": tr, "algorithmic_bytes_per_launch": bytes_per_launch,
                         "points_per_launch": int_pts, "launch_ms": int_ms_max / max(int_n, 1),
                         "interior_share_of_step": int_ms_max / run_ms_max,
                         "volume_stage": {"achieved": stage_achieved, "frac": stage_achieved / peak,
                                          "points_per_launch": vol_pts, "share_of_step": vol_ms_max / run_ms_max,
                                          "note": "all volume kernels of one RK stage (interior, PML slabs, "
                                                  "edges and surface rows); PML auxiliary traffic is not "
                                                  "credited"},
                         "step": {"achieved": value * 1e9 * BYTES_PER_POINT_STEP / 1e9,
                                  "frac": value * BYTES_PER_POINT_STEP / peak}},
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks}
    if ws == 1 and args.workload == "hills" and not args.no_large:
        line["large"] = large_case(peak, setup_free=setup)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # as many full steps from the start as fit in about 30 s: the
        # oracle's steps get slower as the run goes on, so one step would
        # flatter it
        v, th, sample = oracle_rate(prob, 1000, 0, budget_s=30.0)
        line["cpu_baseline"] = {"value": v, "unit": unit, "cores": th, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.finish(ws)


if __name__ == "__main__":
    main()
