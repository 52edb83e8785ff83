"""Benchmark: fused FP32 finite-volume step on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the metric's configuration): 3D Rayleigh-Taylor, compressible
Navier-Stokes at 256^3 over [0,0.5]x[0,0.5]x[0,1.5], FP32 state with FP64
reductions, mu = 1e-4, gravity -0.1 in x3, MUSCL van Leer + HLL + rk3, CFL 0.4
(multiphysics_fvm_b200/setups/rayleigh_taylor_3d.py).  A step is one time step
of the whole grid: device CFL reduction, then per stage the ghost fill and the
fused residual + stage kernel.  Synthetic seeded initial data.

Multi-GPU: the path does not shard (one grid fits one GPU), so N ranks run N
independent replicas ("replicas only"), no data-path collective; the timed
region is the max over ranks of the device time.

--impl reference times the reference algorithm's CPU implementation (the CPU
oracle restatement, since the reference is Python that cannot be installed on
the GPU box) on the host cores: one process per core, each stepping its own
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SIDE = 256
METRIC = "cell-updates/s"
WORKLOAD = ("rayleigh_taylor_3d 256^3 navier_stokes mu=1e-4 g=-0.1 MUSCL van_leer + HLL + rk3, "
            "fp32 state, fp64 dt/totals reductions, CFL 0.4")
# Algorithmic HBM bytes per cell of each rk3 stage launch with a low-storage
# accumulator (R1W2, R3W2, R2W1 field passes of 5 float32 variables; the float32
# kernels move exactly these) and of the dt read.
STAGE_BYTES = [60.0, 100.0, 60.0]
DT_BYTES = 20.0


def reduce_max(dist, value, device="cuda"):
    """Max over ranks of a per-rank duration (identity without a process group)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, cells, steps, seconds):
    """Whole-job cell-updates/s of `world` replicas that each advanced `cells`
    cells `steps` times, with `seconds` the max over ranks."""
    return world * cells * steps / seconds


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def make_state(n, seed=0):
    from multiphysics_fvm_b200.grid.geometry import build_grid
    from multiphysics_fvm_b200.physics import navier_stokes
    from multiphysics_fvm_b200.setups import rayleigh_taylor_3d as rt
    s = rt.get_setup(n, n, n, seed=seed)
    g = build_grid(s["coordinate_system"], s["grid_config"])
    U = navier_stokes.allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
    return s, np.stack([U[k] for k in navier_stokes.VARIABLES])


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.p = None
        self.path = os.path.join(tempfile.gettempdir(), f"fvm_bench_clocks_rank{gpu_index}_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            time.sleep(0.2)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if self.p is None:
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        loaded = [x for x in sm if mx and x > 0.5 * max(mx)] or sm
        return {"sm_mhz": float(np.median(loaded)) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


CPU_N, CPU_STEPS = 96, 3  # about 10 s of one core: large enough that the arrays leave the caches


def cpu_baseline_sample(n=CPU_N, steps=CPU_STEPS):
    """The CPU oracle on a bounded sample of the workload, one core."""
    from oracle import fvm_oracle as O
    s, U = make_state(n)
    geo = O.Geometry("cartesian", s["grid_config"])
    sch = dict(reconstructor="muscl", slope_limiter="van_leer", riemann_solver="hll")
    kinds = [[("periodic", 0.0)] * 4 + [("reflecting" if q == 3 else "neumann", 0.0)] * 2 for q in range(5)]
    bcs = [dict(zip(O.SIDES, k)) for k in kinds]
    O.run("navier_stokes", U, s["physical_parameters"], geo, sch, bcs, "rk3", 0.4, 1)  # warm-up
    t0 = time.perf_counter()
    O.run("navier_stokes", U, s["physical_parameters"], geo, sch, bcs, "rk3", 0.4, steps)
    el = time.perf_counter() - t0
    return n ** 3 * steps / el, el


def _ref_worker(args):
    n, steps, seed = args
    from oracle import fvm_oracle as O
    s, U = make_state(n, seed)
    geo = O.Geometry("cartesian", s["grid_config"])
    sch = dict(reconstructor="muscl", slope_limiter="van_leer", riemann_solver="hll")
    kinds = [[("periodic", 0.0)] * 4 + [("reflecting" if q == 3 else "neumann", 0.0)] * 2 for q in range(5)]
    bcs = [dict(zip(O.SIDES, k)) for k in kinds]
    t0 = time.perf_counter()
    O.run("navier_stokes", U, s["physical_parameters"], geo, sch, bcs, "rk3", 0.4, steps)
    return time.perf_counter() - t0


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = min(os.cpu_count() or 1, 64)
    n = 64  # per-process sample: 64^3 cells of the same setup and schemes (arrays larger than the caches)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_ref_worker, [(n, 1, 100 + i) for i in range(cores)])  # warm-up
        t0 = time.perf_counter()
        pool.map(_ref_worker, [(n, args.steps, i) for i in range(cores)])
        el = time.perf_counter() - t0
    value = cores * n ** 3 * args.steps / el
    line = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "sample": f"{cores} processes x {n}^3 cells (CPU oracle port)"},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                             "sample": f"{cores} x {n}^3 RT cells, {args.steps} steps, NumPy float64"},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def closure_line():
    """Learned closure at 128^3 (tensor cores): forward and training-step device
    times, the tensor roofline of the forward pass, and the KH3D SSPRK3 step
    without/with the closure attached."""
    try:
        import numpy as np
        from multiphysics_fvm_b200 import closure_bench as cb
        r = cb.run(128, 10, np.random.default_rng(0))
        peak, kind = cb.measured_peak()
        return {"grid": [128] * 3, "ms_forward": r["ms_forward"], "ms_train_step": r["ms_train_step"],
                "roofline": {"bound": "tensor", "achieved": r["tflops_forward"], "peak": peak, "unit": "TFLOP/s",
                             "frac": r["tflops_forward"] / peak, "kernel": "conv3_kernel (tcgen05 BF16, forward)",
                             "flop_per_cell": cb.FWD_FLOP, "peak_source": f"bf16_tflops ({kind})"},
                "train_tflops": r["tflops_train"], "ms_step_plain": r["ms_step_plain"],
                "ms_step_closure": r["ms_step_closure"], "status": r["status"]}
    except Exception as e:  # report, never fail the solver bench line
        return {"error": f"{type(e).__name__}: {e}"}


def profile_traffic(name):
    """DRAM bytes per stage launch at 256^3 and their source, from the
    machine-readable lines of a committed ncu summary (profiles/); not measured
    in this run."""
    traffic, source = None, None
    tp = os.path.join(ROOT, "profiles", name)
    if os.path.exists(tp):
        for line in open(tp):
            if "traffic_bytes_per_launch_256:" in line:
                traffic = float(line.split("traffic_bytes_per_launch_256:")[1].split()[0])
            if "traffic_source:" in line:
                source = line.split("traffic_source:")[1].strip().rstrip("->").strip()
    return traffic, source


# North-star kernel: 3D Kelvin-Helmholtz, inviscid, MUSCL minmod + HLL + SSPRK3
# at 256^3 in float32.  SSPRK3 stage launches move R1W1, R2W1, R2W1 field passes
# of 5 float32 variables; the CFL reduction reads the state once.
KH_STAGE_BYTES = [40.0, 60.0, 60.0]


def kh3d_line(steps, warmup, peak, peak_source):
    """Time the fused SSPRK3 MUSCL-HLL step on the 256^3 Kelvin-Helmholtz box
    (setups/kelvin_helmholtz_sharp.py extruded in x3) with CUDA events in the same
    run: ms/step, cell-updates/s, per-launch stage-kernel roofline and the step's
    algorithmic bandwidth at 180 B per cell-update."""
    try:
        from multiphysics_fvm_b200 import run_config
        from multiphysics_fvm_b200.backend import Simulation
        s, U = run_config.make("kh3d", N_SIDE)
        sim = Simulation.from_setup(s)
        sim.upload(U)
        sim.set_time(0.0, math.inf, float(s["time_config"]["CFL"]))
        zchunk, _ = sim.autotune()
        sim.step(warmup)
        ms = sim.time_steps(steps)
        stage_ms, other_ms, launches = sim.profile_steps(max(3, min(steps, 10)))
        status = sim.status()
        tile_ty, _ = sim.tiling()
        sim.close()
        kh_traffic, kh_source = profile_traffic("ns_strip_kh3d_256.md")
        cells = N_SIDE ** 3
        ms_step = ms / steps
        per_launch = stage_ms / launches
        alg_launch = cells * sum(KH_STAGE_BYTES) / len(KH_STAGE_BYTES)
        ach = alg_launch / (per_launch / 1e3) / 1e9
        step_gbs = cells * (sum(KH_STAGE_BYTES) + DT_BYTES) / (ms_step / 1e3) / 1e9
        nst = launches / len(KH_STAGE_BYTES)
        return {"workload": "kelvin_helmholtz 3D 256^3 navier_stokes mu=0, MUSCL minmod + HLL + rk3_ssp, fp32, CFL 0.4",
                "grid": [N_SIDE] * 3, "steps": steps, "ms_per_step": ms_step,
                "value": cells / (ms_step / 1e3), "unit": "cell-updates/s", "device_status": status,
                "tiling": {"tile_rows": tile_ty, "zchunk": zchunk},
                "step_breakdown_ms": {"stage_kernels": stage_ms / nst, "other_kernels": other_ms / nst},
                "step_gbs": step_gbs, "step_frac": step_gbs / peak,
                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                             "traffic": kh_traffic, "traffic_source": kh_source,
                             "kernel": "NS stage kernel (fused residual + SSPRK3 stage)",
                             "per_launch_ms": per_launch, "alg_bytes_per_launch": alg_launch,
                             "bytes_per_cell_update": sum(KH_STAGE_BYTES) + DT_BYTES,
                             "peak_source": peak_source}}
    except Exception as e:  # report, never fail the headline line
        return {"error": f"{type(e).__name__}: {e}"}


def run_ours(args):
    import torch
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from multiphysics_fvm_b200.backend import Simulation
    s, U = make_state(N_SIDE, seed=rank)
    sim = Simulation.from_setup(s)
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.4)
    zchunk, _ = sim.autotune()  # block shape and z-march depth for this grid (state restored)
    tile_rows, _ = sim.tiling()
    step_launches = sim.step_launches()  # the CFL reduction, ghost fills and stage kernels of one step
    cells = N_SIDE ** 3

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    sim.step(args.warmup)
    barrier()
    with ClockSampler(local) as clk:
        ms = sim.time_steps(args.steps)
    barrier()
    ms = reduce_max(dist, ms)
    status = sim.status()
    value = aggregate_rate(world, cells, args.steps, ms / 1e3)

    # dominant kernel: per-launch device time of the stage kernels (events)
    stage_ms, other_ms, launches = sim.profile_steps(max(3, min(args.steps, 10)))
    per_launch_ms = stage_ms / launches
    alg_bytes = cells * sum(STAGE_BYTES) / len(STAGE_BYTES)
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_source = "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650"
    # DRAM bytes per stage launch: not measured in this run; read from the
    # committed ncu capture (profiles/) and labelled with its source
    # the autotuner's two viscous shapes are two kernels: 7-row tiles run the
    # register-blocked kernel, 6-row tiles the general one
    strip = tile_rows == 7
    kernel = ("ns_strip_visc_kernel (register-blocked residual + rk3 stage)" if strip
              else "ns_stage_kernel (fused residual + rk3 stage)")
    traffic, traffic_source = profile_traffic("ns_strip_visc_rt3d_256.md" if strip else "ns_stage_rt3d_256.md")

    # end to end through the public API with host buffers: every step uploads
    # the float64 ghosted state from pinned memory, advances one step and
    # downloads the result; the pipelined calls overlap one step's upload with
    # the previous step's download and compute
    host = torch.from_numpy(U).pin_memory().numpy()
    out = torch.empty(U.shape, dtype=torch.float64).pin_memory().numpy()
    e2e_steps = max(3, min(args.steps, 10))
    sim.upload_async(host)  # first use makes the copy streams and staging buffer
    sim.step_async(1)
    sim.download_async(out)
    sim.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.upload_async(host)
        sim.step_async(1)
        sim.download_async(out)
    sim.synchronize()
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_s = reduce_max(dist, e2e_s)
    e2e = aggregate_rate(world, cells, e2e_steps, e2e_s)

    sim.close()
    kh3d = kh3d_line(args.steps, args.warmup, peak, peak_source) if rank == 0 else None
    if rank == 0:
        cpu_v, cpu_el = cpu_baseline_sample()
        closure = closure_line()
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded RT initial state)",
            "config": {"workload": WORKLOAD, "grid": [N_SIDE] * 3, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (each state buffer 345 MB > 126 MB)",
                       "timing": "CUDA events on the handle stream around K graph launches, max over ranks",
                       "tile_rows": tile_rows, "zchunk": zchunk},
            # per step (fvm_step_launches): the CFL reduction, then per stage a
            # ghost fill (the first one also closes the clock) and the stage kernel
            "gpu_launches": args.steps * step_launches,
            "device_status": status,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_source,
                         "kernel": kernel,
                         "per_launch_ms": per_launch_ms, "alg_bytes_per_launch": alg_bytes,
                         "peak_source": peak_source},
            "step_breakdown_ms": {"stage_kernels": stage_ms / (launches / len(STAGE_BYTES)),
                                  "other_kernels": other_ms / (launches / len(STAGE_BYTES))},
            "e2e": {"value": e2e, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": int(U.nbytes), "d2h_bytes_per_step": int(U.nbytes),
                    "how": "fvm_upload_async(pinned float64 state) + fvm_step_async(1) + fvm_download_async per "
                           "step, pipelined on two copy streams, wall clock to fvm_synchronize"},
            "cpu_baseline": {"value": cpu_v, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                             "sample": f"CPU oracle, {CPU_N}^3 RT cells, {CPU_STEPS} rk3 steps ({cpu_el:.1f} s), "
                                       "NumPy float64"},
            "clocks": clk.summary(),
            "closure": closure,
            "kh3d_ssprk3_256": kh3d,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
