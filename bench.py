"""Benchmark of the fused Euler step on B200.

Workload: 3D Sod shock tube on a 512^3 grid (plus 2 ghost layers), FP32
conserved state (rho, rho*u, rho*v, rho*w, E) in HBM, gamma 1.4, minmod
slopes, CFL 0.4, outflow boundaries.  One bench step = one call of the
reference's compute_step = one launch of the fused kernel over all 512^3
cells.  Data: synthetic (the workload's initial state, built on the GPU).

Metric: GCUPS = 1e9 cell updates per second (whole job: all ranks).

Keys beside the contract's ones:
  roofline      the step against measured HBM bandwidth: achieved = 40 B
                per cell update (read + write 5 FP32 fields) x cells / mean
                step time (CUDA events on the library's stream; a step is the
                interior-tile launch and the frame launch that overlaps its
                last wave); traffic = ncu DRAM bytes per step from the
                committed profile of the same kernel pair
                (profiles/step_traffic.json), else null.
  e2e           the same metric through the C ABI from pinned HOST buffers:
                upload of the state, K steps reading dt back after each one
                (as the reference's time loop does), download of the state.
  cpu_baseline  the C oracle (a restatement of the reference's Rust step)
                on the host cores, bounded sample of the same workload;
                OpenMP over every loop, and under "rust_like" threaded only
                where the Rust step is (its serial loops stay serial).
  clocks        nvidia-smi samples during the timed region.
  vortex        the workload's second case, the 512^3 isentropic vortex
                (periodic), timed the same way (GCUPS, ms per step).
  parity        per-field relative L1 of the FP32 step against the FP64
                oracle after 20 steps of Sod and of the vortex at 128^3, and
                the relative difference of the last dt (computed with the
                CPU baseline, outside every timed region).

--case learned: the learned coarse-grid correction end to end -- training
pairs made by the solver (256^3 fine / 128^3 coarse), 2000 Adam steps of the
tensor-core network, then held-out KH and Fourier states solved by every
method (plain 512^3, 256^3, 128^3, 64^3; corrected 256^3 and 128^3) to the
time the 512^3 grid reaches in 400 steps, against a plain 1024^3 solve as
the truth.  Metric: time to a relative L1 density error <= 2 % (fastest
method); beside it every method's error and time, the workload's criterion
(corrected 256^3 within 1.5x of the 512^3 error), the 512^3 / corrected
256^3 time ratio and the network's forward throughput against the measured
BF16 peak.  Takes a few minutes.

--case netfwd: the correction network's forward pass alone (4 tcgen05 BF16
convolutions, random weights) on an (n+8)^3 input, as the corrector runs it
on an n^3 grid; TFLOP/s against the measured BF16 peak.

--case corrector: one corrected coarse step (plain step, network, checked
correction) on an n^3 periodic KH state with random network weights.

--case snapshot: the state output of the reference's time loop
(save_to_disk, io.rs:5-196) for the 512^3 state: capture time on the step
stream, device->host copy rate, the step time while a copy is in flight,
and the file write rate.

--case refcuda: the reference's own CUDA solver on the same GPU, as the
same-box comparator.  oracle/refcu builds its src/cu sources (physics.hpp's
compute_step and kernels, unchanged; spdlog, HighFive and NVTX stubbed) for
sm_100a on its TRB configuration header (ini_files/trb.h: 124 x 124 x 252
interior cells, walls, gravity, FP32); that program sets up the reference's
own rising-bubble state, runs its stock time step and reports its time.
This library then steps the same state on the same configuration: the
first step is compared field by field with the reference's, and K steps
are timed both as one enqueued sequence (device time) and as the
reference's loop runs (one call per step, dt read back each step).

--impl reference times the reference's CPU algorithm (the oracle port; the
Rust crate cannot be built on this image) on the same workload and metric.
Multi-GPU (torchrun): independent replicas, one 512^3 grid per rank
(the step has no exchange in this configuration); timing is the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "deep-green_b200" / "python"))

METRIC = "GCUPS"
UNIT = "1e9 cell-updates/s"
GAMMA, CFL = 1.4, 0.4
BYTES_PER_CELL = {"f32": 40, "f64": 80}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512, help="interior cells per axis")
    ap.add_argument("--case", default="sod", choices=["sod", "vortex", "batch64", "learned", "netfwd", "snapshot", "corrector",
                                                          "refcuda"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def job_rate(ms_local, cells_per_rank, steps, world, device=None):
    """Whole-job rate of `world` independent replicas: all ranks' cell
    updates over the slowest rank's device time (all_reduce MAX, the same
    collective on every rank).  Returns (GCUPS, max ms)."""
    ms = float(ms_local)
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return world * cells_per_rank * steps / (ms * 1e-3) / 1e9, ms


def workload_name(case, n):
    return f"{case}3d_{n}^3_fp32_minmod_cfl{CFL}"


# --------------------------------------------------------------------------
# GPU set-up of the initial state (conserved totals, ghosted, dense)
# --------------------------------------------------------------------------
def device_initial_state(case, n, device):
    import torch
    f64 = torch.float64
    m = n + 4
    if case == "sod":
        ds = 1.0 / n
        x = (torch.arange(m, dtype=f64, device=device) - 2 + 0.5) * ds
        left = (x < 0.5).view(m, 1, 1).expand(m, m, m)
        rho = torch.where(left, 1.0, 0.125).to(f64)
        p = torch.where(left, 1.0, 0.1).to(f64)
        vx = torch.zeros((m, m, m), dtype=f64, device=device)
        vy = torch.zeros_like(vx)
        vz = torch.zeros_like(vx)
        bcs = (1,) * 6
    else:
        L, beta = 5.0, 5.0
        ds = 2 * L / n
        c = -L + (torch.arange(m, dtype=f64, device=device) - 2 + 0.5) * ds
        x = c.view(m, 1, 1)
        y = c.view(1, m, 1)
        r2 = x * x + y * y
        e = torch.exp(0.5 * (1 - r2))
        T = 1 - (GAMMA - 1) * beta * beta / (8 * GAMMA * np.pi ** 2) * e * e
        rho = (T ** (1 / (GAMMA - 1))).expand(m, m, m).contiguous()
        p = rho ** GAMMA
        vx = (1 - beta / (2 * np.pi) * e * y).expand(m, m, m).contiguous()
        vy = (1 + beta / (2 * np.pi) * e * x).expand(m, m, m).contiguous()
        vz = torch.zeros((m, m, m), dtype=f64, device=device)
        bcs = (0,) * 6
    V = ds * ds * ds
    cons = [rho * V, vx * rho * V, vy * rho * V, vz * rho * V,
            V * (rho * (vx * vx + vy * vy + vz * vz) / 2 + p / (GAMMA - 1))]
    cons = [c.to(torch.float32).contiguous() for c in cons]
    return cons, ds, bcs


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        # start sampling and wait for the first sample, so that the whole
        # timed region is covered (nvidia-smi takes ~0.1-0.5 s to start)
        self.lines = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.skip = len(self.lines)          # samples taken before the timed region
        return self

    def _read(self):
        for l in self.proc.stdout:
            if l.strip():
                self.lines.append(l)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self.reader.join(timeout=5)
            # keep the last pre-region sample (taken within 20 ms of the start) and all later ones
            self.lines = self.lines[max(self.skip - 1, 0):]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU oracle timing (reference algorithm on the host cores)
# --------------------------------------------------------------------------
def cpu_oracle_gcups(case, n, nz_sample, steps, warmup=1, rust_like=False):
    """GCUPS of the C oracle in FP32 on an n x n x nz_sample slab: OpenMP over
    every loop, or (rust_like) parallel only where the Rust step uses
    par_for_each (calc_primitives, calc_timestep, calc_gradients) and serial
    elsewhere, as the reference binary runs."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from deepgreen import setups
    if case == "sod":
        prim, ds, bcs = setups.sod(n, ny=n, nz=nz_sample)
    else:
        prim, ds, bcs = setups.isentropic_vortex(n, ny=n, nz=nz_sample)
    o = pyoracle.Oracle((n, n, nz_sample), ds, bcs, gamma=GAMMA, cfl=CFL, limiter=1, dtype=np.float32,
                        threads=pyoracle.RUST_LIKE if rust_like else pyoracle.ALL_PARALLEL)
    o.set_primitives([a.astype(np.float32) for a in prim])
    del prim
    if warmup:
        o.step(warmup)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        o.step(1)
        times.append(time.perf_counter() - t)
    o.close()
    cells = n * n * nz_sample
    return cells / statistics.mean(times) / 1e9, times


def ncu_traffic_per_step(kernel, n):
    """DRAM bytes per step of the benchmarked kernel pair, from the committed
    ncu summary (profiles/step_traffic.json): only when that capture is of
    the same kernels; each launch's bytes per cell scaled to its own cells on
    an n^3 grid (interior tiles: full 14 x 64 tiles two cells clear of every
    y and z face; the frame: the rest).  None otherwise."""
    p = ROOT / "profiles" / "step_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        if d["kernel"] != kernel:
            return None
        ny_in, nz_in = (n - 2) // 14 - 1, (n - 2) // 64 - 1
        interior = ny_in * 14 * nz_in * 64 * n if ny_in > 0 and nz_in > 0 else 0
        return float(d["interior_bytes_per_cell"]) * interior + float(d["frame_bytes_per_cell"]) * (n ** 3 - interior)
    except Exception:
        return None


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
def run_reference(args, world, rank):
    if rank != 0:
        return
    n = args.n
    nz_sample = 64
    cores = os.cpu_count()
    gcups, times = cpu_oracle_gcups(args.case, n, nz_sample, args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": gcups, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args.case, n), "grid": [n, n, n], "ghosts": 2,
                   "parallelism": f"host CPU, {cores} threads", "sample": f"{n}x{n}x{nz_sample} slab of the grid"},
        "cpu_baseline": {"value": gcups, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} steps of a {n}x{n}x{nz_sample} slab, same physics, FP32, "
                                   f"C restatement of the Rust step, OpenMP over {cores} threads"},
        "e2e": {"value": gcups, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# The step's launches on grids with interior tiles (512^3: 71 % of the
# tiles): the interior tiles, then the frame of tiles along the y and z faces.
STEP_KERNEL = ("dg::sweep::sweep_step_kernel<float, 14, 4, 1, false, true> + "
               "dg::sweep::sweep_step_kernel<float, 14, 4, 1, false, false>")


def step_launches(n, ny=None, nz=None):
    """Launches per step of the FP32 sweep on an n x ny x nz grid (ny, nz
    default to n): two with interior tiles (full 14 x 64 tiles two cells
    clear of every y and z face), else one."""
    ny_in = ((n if ny is None else ny) - 2) // 14 - 1
    nz_in = ((n if nz is None else nz) - 2) // 64 - 1
    return 2 if ny_in > 0 and nz_in > 0 else 1


def timed_steps(ctx, steps, warmup, local, world, barrier):
    """K steps of the context's kernel timed with CUDA events on its stream
    (max over ranks), with the clock samples of the timed region."""
    import torch
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    ctx.enqueue_steps(warmup)
    ctx.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        ctx.enqueue_steps(steps)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    barrier()
    return start.elapsed_time(end), clk.summary()


def parity_block(n=128, steps=20):
    """Per-field relative L1 (sum|a-b| / sum|b| over the interior) of the FP32
    production kernel against the FP64 oracle after `steps` steps of the Sod
    and vortex workloads at n^3 (a size the oracle runs in about a second),
    and the relative difference of the last dt.  Part of the CPU-baseline leg:
    the oracle is the checker here, nothing of it is timed or shipped."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from deepgreen import capi, setups
    out = {"grid": [n, n, n], "steps": steps, "against": "FP64 oracle (C restatement of the Rust step)",
           "tolerance": 1e-5}
    for case in ("sod", "vortex"):
        if case == "sod":
            prim, ds, bcs = setups.sod(n)
        else:
            prim, ds, bcs = setups.isentropic_vortex(n, gamma=GAMMA)
        o = pyoracle.Oracle((n, n, n), ds, bcs, gamma=GAMMA, cfl=CFL, limiter=1, dtype=np.float64,
                            threads=pyoracle.ALL_PARALLEL)
        o.set_primitives([np.asarray(a, np.float64) for a in prim])
        odts = o.step(steps)
        ref = o.conserved()
        o.close()
        ctx = capi.Context((n, n, n), ds, bcs, gamma=GAMMA, cfl=CFL, limiter=capi.LIMITER_MINMOD,
                           precision=capi.F32)
        ctx.set_primitives([np.asarray(a, np.float32) for a in prim])
        gdts = ctx.compute_step(steps)
        got = ctx.get_conserved()
        ctx.close()
        inner = (slice(2, -2),) * 3
        errs = {}
        for f, name in enumerate(("mass", "mom_x", "mom_y", "mom_z", "energy")):
            b = np.asarray(ref[f], np.float64)[inner]
            a = np.asarray(got[f], np.float64)[inner]
            den = np.abs(b).sum()
            # a field that is zero in the reference (the Sod tube's transverse
            # momenta) is reported as the absolute L1 over the mass's scale
            errs[name] = float(np.abs(a - b).sum() / den) if den > 0 else \
                float(np.abs(a - b).sum() / np.abs(np.asarray(ref[0], np.float64)[inner]).sum())
        out[case] = {"rel_l1": errs, "max": max(errs.values()),
                     "dt_rel": float(abs(gdts[-1] - odts[-1]) / odts[-1])}
    out["kh64"] = kh64_block()
    return out


def kh64_block(steps=200):
    """The 64^3 Kelvin-Helmholtz workload (periodic, gamma 1.4, minmod, CFL
    0.4), 200 steps: per-field relative L1 of the FP32 production kernel and
    of the reference's own f32 arithmetic (the oracle's float instantiation)
    against the FP64 oracle.  The transverse momenta are noise-level fields
    that the instability amplifies, where both FP32 results drift from FP64
    far beyond 1e-5; the parity test bounds them by twice the reference f32
    error."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from deepgreen import capi, setups
    prim, ds, bcs = setups.kelvin_helmholtz(64, seed=1)
    shape = (64, 64, 64)
    res = {}
    for dtype in (np.float64, np.float32):
        o = pyoracle.Oracle(shape, ds, bcs, gamma=GAMMA, cfl=CFL, limiter=1, dtype=dtype,
                            threads=pyoracle.ALL_PARALLEL)
        o.set_primitives([np.asarray(a, dtype) for a in prim])
        o.step(steps)
        res[dtype] = o.conserved()
        o.close()
    ctx = capi.Context(shape, ds, bcs, gamma=GAMMA, cfl=CFL, limiter=capi.LIMITER_MINMOD, precision=capi.F32)
    ctx.set_primitives([np.asarray(a, np.float32) for a in prim])
    ctx.compute_step(steps)
    got = ctx.get_conserved()
    ctx.close()
    inner = (slice(2, -2),) * 3
    names = ("mass", "mom_x", "mom_y", "mom_z", "energy")

    def rel(a, f):
        b = np.asarray(res[np.float64][f], np.float64)[inner]
        return float(np.abs(np.asarray(a, np.float64)[inner] - b).sum() / np.abs(b).sum())
    return {"steps": steps, "kernel_fp32": {n: rel(got[f], f) for f, n in enumerate(names)},
            "reference_f32_arithmetic": {n: rel(res[np.float32][f], f) for f, n in enumerate(names)}}


def run_ours(args, world, rank, local):
    import torch
    from deepgreen import capi
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def make(case):
        cons, ds, bcs = device_initial_state(case, n, dev)
        c = capi.Context((n, n, n), ds, bcs, gamma=GAMMA, cfl=CFL, limiter=capi.LIMITER_MINMOD,
                         precision=capi.F32, device=local)
        torch.cuda.synchronize()   # the fields are complete before the library's stream copies them
        c.set_conserved_device([x.data_ptr() for x in cons])
        return c, cons

    ctx, cons = make(args.case)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    blocks, threads, chunk = ctx.launch_shape()
    ms, clocks = timed_steps(ctx, args.steps, args.warmup, local, world, barrier)
    dts = ctx.get_dts(args.steps)
    status = ctx.status()
    cells = n ** 3
    value, ms = job_rate(ms, cells, args.steps, world, device=dev)
    ms_step = ms / args.steps

    # end to end through the C ABI from pinned host buffers
    e2e = None
    if not args.no_e2e:
        host_in = [c.cpu().pin_memory() for c in cons]
        host_out = [torch.empty_like(h).pin_memory() for h in host_in]
        ptr_in = [h.data_ptr() for h in host_in]
        ptr_out = [h.data_ptr() for h in host_out]
        import ctypes
        lib = ctx.lib
        arr_in = (ctypes.c_void_p * 5)(*ptr_in)
        arr_out = (ctypes.c_void_p * 5)(*ptr_out)
        dtbuf = (ctypes.c_double * 1)()
        # warm-up of the path (untimed): the first copies from freshly pinned
        # pages run slower than the link
        ctx._check(lib.dg_set_conserved(ctx.h, arr_in))
        ctx._check(lib.dg_compute_step(ctx.h, 1, dtbuf))
        ctx._check(lib.dg_get_conserved(ctx.h, arr_out))
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx._check(lib.dg_set_conserved(ctx.h, arr_in))
        for _ in range(args.steps):
            ctx._check(lib.dg_compute_step(ctx.h, 1, dtbuf))
        ctx._check(lib.dg_get_conserved(ctx.h, arr_out))
        e1.record(stream)
        e1.synchronize()
        barrier()
        e2e_value, e2e_ms = job_rate(e0.elapsed_time(e1), cells, args.steps, world, device=dev)
        state_bytes = 5 * (n + 4) ** 3 * 4
        e2e = {"value": e2e_value, "unit": UNIT,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps + 8,
               "ms_total": e2e_ms, "path": "dg_set_conserved + K x dg_compute_step(1) + dg_get_conserved"}
        del host_in, host_out
    del cons
    ctx.close()

    # the workload's second case: the 512^3 isentropic vortex (periodic)
    other = None
    if args.case == "sod":
        vctx, vcons = make("vortex")
        del vcons
        vms, vclk = timed_steps(vctx, args.steps, args.warmup, local, world, barrier)
        vvalue, vms = job_rate(vms, cells, args.steps, world, device=dev)
        vctx.close()
        other = {"workload": workload_name("vortex", n), "value": vvalue, "unit": UNIT,
                 "ms_per_step": vms / args.steps, "clocks": vclk}

    if rank != 0:
        return
    peak, peak_kind = peaks()
    achieved = BYTES_PER_CELL["f32"] * cells / (ms_step * 1e-3) / 1e9
    traffic = ncu_traffic_per_step(STEP_KERNEL, n)
    cpu = None
    parity = None
    if not args.no_cpu and world == 1:
        nz_sample = 64
        g, times = cpu_oracle_gcups(args.case, n, nz_sample, 5, warmup=1)
        cpu = {"value": g, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"5 steps of a {n}x{n}x{nz_sample} slab of the same workload (FP32, C restatement "
                         f"of the Rust step, OpenMP over all host threads)"}
        # the same restatement threaded as the Rust binary is (its serial
        # loops stay serial): the stand-in for the reference's own speed
        g_rust, _ = cpu_oracle_gcups(args.case, n, 16, 2, warmup=1, rust_like=True)
        cpu["rust_like"] = {"value": g_rust, "unit": UNIT,
                            "sample": f"2 steps of a {n}x{n}x16 slab; threads only where the Rust step "
                                      f"uses par_for_each (calc_primitives, calc_timestep, calc_gradients)"}
        parity = parity_block()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args.case, n), "grid": [n, n, n], "ghosts": 2,
                   "parallelism": f"replicas x{world}" if world > 1 else "single grid",
                   "l2": "state (2.9 GB read + 2.9 GB written per step) is larger than L2",
                   "kernel": STEP_KERNEL,
                   "launch": {"blocks": blocks, "threads": threads, "x_planes_per_block": chunk}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": BYTES_PER_CELL["f32"] * cells,
                     "launches_per_step": step_launches(n)},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        "gpu_launches": step_launches(n) * args.steps,
        "dt_first_last": [float(dts[0]), float(dts[-1])],
        "status_flags": status,
    }
    if other:
        line["vortex"] = other
    if parity:
        line["parity"] = parity
    print(json.dumps(line), flush=True)


def run_batch(args, world, rank, local):
    """64 independent grids (edges log-uniform in [32, 160] per axis, seeded),
    each a random two-state Riemann problem, FP32, per-grid CFL dt, one
    persistent launch per step replayed from a CUDA graph, tiling chosen by
    the autotuner.  Timed twice: with each grid stored in the axis order that
    pads its tiles least (DG_BATCH_REORIENT, the line's value) and in the
    callers' order (caller_layout)."""
    import torch
    from deepgreen import batch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shapes = batch.grid_shapes(64, 32, 160, seed=2024)
    cells = sum(a * b * c for a, b, c in shapes)

    def fill(bt):
        # updated cells / cells the kernel's tiles cover (z padded to 64
        # columns, y to the tile rows), over the stored orientations
        padded = 0
        rows = bt.tiling()[0]
        for i, sh in enumerate(shapes):
            nx, ny, nz = (sh[a] for a in bt.orientation(i))
            padded += nx * -(-ny // rows) * rows * -(-nz // 64) * 64
        return cells / padded

    def timed(reorient):
        bt, specs, prims = batch.make_batch(shapes, seed=2024, device=local, reorient=reorient)
        del prims
        rows, chunk, tune_ms, cached = batch.tuned(bt, shapes, torch.cuda.get_device_name(local),
                                                   reorient=reorient)
        stream = torch.cuda.ExternalStream(bt.stream(), device=dev)
        bt.step(args.warmup)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            start.record(stream)
            bt.enqueue(args.steps)
            end.record(stream)
            end.synchronize()
        ms = start.elapsed_time(end)
        value, ms = job_rate(ms, cells, args.steps, world, device=dev)
        r, c, items = bt.tiling()
        out = {"value": value, "ms_per_step": ms / args.steps, "tile_rows": r, "x_planes_per_item": c,
               "items": items, "tuning_cached": cached, "tile_fill": fill(bt), "clocks": clk.summary()}
        bt.close()
        return out

    caller = timed(False)
    reo = timed(True)
    if rank != 0:
        return
    peak, peak_kind = peaks()
    ms_step = reo["ms_per_step"]
    achieved = BYTES_PER_CELL["f32"] * cells / (ms_step * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": reo["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch64_riemann_fp32_minmod_cfl0.4", "grids": len(shapes), "cells": cells,
                   "layout": "reoriented (DG_BATCH_REORIENT)", "tile_rows": reo["tile_rows"],
                   "x_planes_per_item": reo["x_planes_per_item"], "items": reo["items"],
                   "tile_fill": reo["tile_fill"], "tuning_cached": reo["tuning_cached"],
                   "l2": "state (1.1 GB read + written per step) is larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind},
        "caller_layout": {k: caller[k] for k in ("value", "ms_per_step", "tile_fill", "x_planes_per_item", "items")},
        "clocks": reo["clocks"], "gpu_launches": args.steps,
    }
    print(json.dumps(line), flush=True)


def run_learned(args, world, rank, local):
    """Learned coarse-grid correction: train on solver pairs, then solve
    held-out KH and Fourier states with every method (plain 512^3, 256^3,
    128^3, 64^3; corrected 256^3 and 128^3) to the time the 512^3 grid
    reaches in 400 steps, against a plain 1024^3 solve as the truth
    (rank 0; other ranks idle).  Metric: time to a solution whose relative L1
    density error is <= 2 %, fastest method; beside it every method's error
    and time, the workload's criterion (corrected 256^3 within 1.5x of the
    512^3 error) and the 512^3 / corrected 256^3 time ratio."""
    import torch
    from deepgreen import learned, learned_workload as lw
    if rank != 0:
        return
    torch.cuda.set_device(local)
    quiet = lambda *a: None  # noqa: E731
    traj = [("kh", 100 + i) for i in range(8)] + [("fourier", 200 + i) for i in range(8)]
    net, norm, ps, tr = lw.training(128, traj, 8, 20, 40, 2000, 8, 64, 1e-3, 0, log=quiet)
    del ps
    torch.cuda.empty_cache()
    cases = [lw.evaluate_truth(net, norm, "kh", 9001, 256, 400, log=quiet, train_n=128, shear=0.5, ratio=2.0),
             lw.evaluate_truth(net, norm, "fourier", 9002, 256, 400, log=quiet, train_n=128)]
    # the network alone at the corrector's shape: 264^3 input -> 256^3 fluxes
    dev = torch.device("cuda", local)
    feat = torch.zeros((1, 264, 264, 264, 16), dtype=torch.bfloat16, device=dev)
    feat[..., :learned.INPUTS] = torch.randn((1, 264, 264, 264, learned.INPUTS), device=dev).to(torch.bfloat16)
    out = net.forward(feat)
    net.synchronize()
    stream = torch.cuda.ExternalStream(net.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        net.forward(feat, out)
    e1.record(stream)
    net.synchronize()
    fwd_ms = e0.elapsed_time(e1) / 5
    flop = 2 * 27 * (learned.INPUTS * 32 + 32 * 32 * 2 + 32 * learned.OUTPUTS) * 256 ** 3
    pk = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(pk.get("bf16_tflops", 1590.0))
    achieved = flop / (fwd_ms * 1e-3) / 1e12
    fastest = [c["time_to_l1"]["fastest_seconds"] for c in cases]
    value = max(fastest) if all(f is not None for f in fastest) else None
    line = {
        "metric": "time to L1(rho) <= 2 % (fastest method, slower of the two cases)", "value": value,
        "unit": "s", "n_gpus": 1, "steps": 400, "warmup": 2, "higher_is_better": False, "scaling": "none",
        "vs_baseline": None, "dtype": "bf16 network, f32 state", "data": "synthetic",
        "config": {"workload": "learned_correction_256_vs_512", "train": "128^3/256^3 pairs, 2000 x 8 crops of 64^3",
                   "horizon": "time of 400 steps of the 512^3 grid", "truth": "plain 1024^3 FP32 solve"},
        "learned": {"training": {k: v for k, v in tr.items() if k != "loss_history"},
                    "cases": [{k: c[k] for k in ("kind", "t_end", "l1_density", "l1_density_plain_512_at_256",
                                                  "seconds", "steps", "corrector",
                                                  "criterion_learned_within_1p5x_of_plain_512",
                                                  "time_ratio_plain_512_over_learned_256", "time_to_l1",
                                                  "by_method_at_256")}
                              for c in cases]},
        "time_ratio_plain_512_over_learned_256": [c["time_ratio_plain_512_over_learned_256"] for c in cases],
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel": "network forward at 264^3 (4 tcgen05 convolutions), algorithmic FLOP"},
    }
    print(json.dumps(line), flush=True)


def run_netfwd(args, world, rank, local):
    """The correction network's forward pass alone at the corrector's shape."""
    import torch
    from deepgreen import learned
    from deepgreen.net import Net
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    net = Net(learned.INPUTS, learned.OUTPUTS, seed=1, out_scale=0.1)
    feat = torch.zeros((1, n + 8, n + 8, n + 8, 16), dtype=torch.bfloat16, device=dev)
    feat[..., :learned.INPUTS] = torch.randn((1, n + 8, n + 8, n + 8, learned.INPUTS), device=dev).to(torch.bfloat16)
    out = net.forward(feat)
    for _ in range(max(args.warmup - 1, 0)):
        net.forward(feat, out)
    net.synchronize()
    stream = torch.cuda.ExternalStream(net.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            net.forward(feat, out)
        e1.record(stream)
        net.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    flop = 2 * 27 * (learned.INPUTS * 32 + 32 * 32 * 2 + 32 * learned.OUTPUTS) * n ** 3
    pk = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(pk.get("bf16_tflops", 1590.0))
    achieved = flop / (ms * 1e-3) / 1e12
    line = {
        "metric": "network forward TFLOP/s", "value": achieved, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "none", "vs_baseline": None,
        "dtype": "bf16", "data": "synthetic",
        "config": {"workload": f"correction_network_forward_{n}^3", "input": f"{n + 8}^3 x 16 ch",
                   "layers": "15-32-32-32-15, 3x3x3", "flop_per_cell": flop // n ** 3},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": "measured" if pk else "fallback"},
        "clocks": clk.summary(), "gpu_launches": 4 * args.steps,
    }
    print(json.dumps(line), flush=True)


def run_snapshot(args, world, rank, local):
    """Snapshot output (save_to_disk, io.rs:5-196) of the n^3 Sod state: the
    capture's cost on the step stream, the device->host copy rate, the step
    time while a copy is in flight, and the file write rate."""
    import tempfile
    import torch
    from deepgreen import capi, snapshot
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    cons, ds, bcs = device_initial_state("sod", n, dev)
    ctx = capi.Context((n, n, n), ds, bcs, gamma=GAMMA, cfl=CFL, limiter=capi.LIMITER_MINMOD,
                       precision=capi.F32, device=local)
    torch.cuda.synchronize()   # the fields are complete before the library's stream copies them
    ctx.set_conserved_device([c.data_ptr() for c in cons])
    del cons
    ctx.enqueue_steps(max(args.warmup, 1))
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    snap = snapshot.Snapshot(ctx)
    nbytes = 10 * (n + 4) ** 3 * 4
    snap.begin()
    snap.wait()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    captures, copies = [], []
    for _ in range(3):
        ctx.synchronize()
        ev[0].record(stream)
        t0 = time.perf_counter()
        snap.begin()
        ev[1].record(stream)
        snap.wait()
        copies.append(time.perf_counter() - t0)
        ev[1].synchronize()
        captures.append(ev[0].elapsed_time(ev[1]))
    k = 10
    ctx.synchronize()
    ev[0].record(stream)
    ctx.enqueue_steps(k)
    ev[1].record(stream)
    ev[1].synchronize()
    plain_ms = ev[0].elapsed_time(ev[1]) / k
    snap.begin()
    ev[2].record(stream)
    ctx.enqueue_steps(k)
    ev[3].record(stream)
    ev[3].synchronize()
    snap.wait()
    overlapped_ms = ev[2].elapsed_time(ev[3]) / k
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "state.00000.dgsnap")
        t0 = time.perf_counter()
        snap.write(path)
        write_s = time.perf_counter() - t0
        size = os.path.getsize(path)
    snap.close()
    cap = statistics.median(captures)
    line = {
        "metric": "snapshot capture time on the step stream", "value": cap, "unit": "ms",
        "n_gpus": 1, "steps": k, "warmup": args.warmup, "higher_is_better": False, "scaling": "none",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"snapshot_sod_{n}^3_fp32", "groups": "primitives + conserved", "bytes": nbytes},
        # capture traffic: read 2 states (5 fields each), write 10 dense fields
        "capture_GBps": 2 * nbytes / (cap * 1e-3) / 1e9,
        "d2h_GBps": nbytes / statistics.median(copies) / 1e9,
        "step_ms": plain_ms, "step_ms_during_copy": overlapped_ms,
        "file_write_GBps": size / write_s / 1e9,
        "gpu_launches": 1,
    }
    print(json.dumps(line), flush=True)


def run_corrector(args, world, rank, local):
    """One corrected coarse step (plain step + the correction network + the
    checked correction) on an n^3 periodic KH state, random network weights:
    the per-step cost of the learned workload's coarse solve."""
    import torch
    from deepgreen import learned
    from deepgreen.net import Net
    if rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    prim, _ = learned.initial_state("kh", n, 5, shear=0.5, ratio=2.0)
    g = learned.grid(n, device=local)
    g.set_primitives(prim)
    del prim
    net = Net(learned.INPUTS, learned.OUTPUTS, seed=0, out_scale=0.01)
    norm = learned.Norm.identity()
    for c in range(5):
        norm.out_std[c] = 1e-4
    for c in range(14, 16):
        norm.in_inv_std[c] = 0.0
    cor = learned.Corrector(g, net, norm)
    cor.step(args.warmup)
    g.synchronize()
    stream = torch.cuda.ExternalStream(g.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        cor.step(args.steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    st = cor.stats()
    cor.close()
    line = {
        "metric": "corrected coarse step time", "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "none", "vs_baseline": None,
        "dtype": "bf16 network, f32 state", "data": "synthetic",
        "config": {"workload": f"corrected_step_kh_{n}^3", "network": "14-32-32-32-15, 3x3x3, random weights"},
        "fallback_steps": st["fallback_steps"], "clocks": clk.summary(), "gpu_launches": 9 * args.steps,
    }
    print(json.dumps(line), flush=True)


REFCUDA = ROOT / "oracle" / "_ref" / "refcu" / "refcu_gpu_trb"
# ini_files/trb.h, as the program built from it reports it
TRB = {"n": (128, 128, 256), "ds": 1.0, "gamma": float(np.float32(5.0 / 3.0)), "cfl": float(np.float32(0.2)),
       "g": float(np.float32(-9.81))}


def run_refcuda(args, world, rank, local):
    """The reference's CUDA solver (built from its sources for this GPU) and
    this library on the reference's TRB configuration, same state, same GPU."""
    if rank != 0:
        return
    import ctypes
    import tempfile

    import torch
    from deepgreen import capi
    base = {"case": "refcuda", "metric": METRIC, "unit": UNIT}
    if not REFCUDA.exists():
        print(json.dumps({**base, "unavailable": "oracle/_ref/refcu/refcu_gpu_trb not built "
                          "(make -C oracle/refcu needs the reference sources)"}), flush=True)
        return
    torch.cuda.set_device(local)
    n = TRB["n"]
    cells = int(np.prod(n))
    interior = tuple(k - 4 for k in n)
    with tempfile.TemporaryDirectory() as d:
        state = Path(d) / "state.bin"
        with ClockSampler(local) as rclk:
            out = subprocess.run([str(REFCUDA), str(max(args.warmup, 1)), str(args.steps), str(state)],
                                 capture_output=True, text=True, timeout=900)
        if out.returncode != 0:
            print(json.dumps({**base, "unavailable": f"reference program exited {out.returncode}: "
                              f"{out.stderr.strip()[-200:]}"}), flush=True)
            return
        ref = json.loads(out.stdout.strip().splitlines()[-1])
        raw = state.read_bytes()
    fields = cells * 4
    prim = [np.frombuffer(raw[f * fields:(f + 1) * fields], np.float32).reshape(n) for f in range(5)]
    ref_dt1 = float(np.frombuffer(raw[5 * fields:5 * fields + 8], np.float64)[0])
    off = 5 * fields + 8
    ref_cons = [np.frombuffer(raw[off + f * fields:off + (f + 1) * fields], np.float32).reshape(n)
                for f in range(5)]
    walls = (2,) * 6
    ctx = capi.Context(interior, TRB["ds"], walls, gamma=TRB["gamma"], cfl=TRB["cfl"], g=TRB["g"], gravity=True,
                       limiter=capi.LIMITER_NONE, precision=capi.F32, device=local)
    ctx.set_primitives(prim)
    dt1 = float(ctx.compute_step(1)[0])
    got = ctx.get_conserved()
    # every interior cell but the first layer at each wall, where the CUDA
    # variant (no ghost rules for its derived arrays) and the Rust path differ
    reg = (slice(3, n[0] - 3), slice(3, n[1] - 3), slice(3, n[2] - 3))
    names = ("mass", "mom_x", "mom_y", "mom_z", "energy")
    errs = {}
    for f, nm in enumerate(names):
        a = np.asarray(got[f], np.float64)[reg]
        b = np.asarray(ref_cons[f], np.float64)[reg]
        den = np.abs(b).sum()
        errs[nm] = float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())
    # timing from the reference's initial state again
    ctx.set_primitives(prim)
    ms, clocks = timed_steps(ctx, args.steps, max(args.warmup, 1), local, 1, lambda: None)
    ctx.set_primitives(prim)
    dtbuf = (ctypes.c_double * 1)()
    for _ in range(max(args.warmup, 1)):
        ctx._check(ctx.lib.dg_compute_step(ctx.h, 1, dtbuf))
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx._check(ctx.lib.dg_compute_step(ctx.h, 1, dtbuf))
    e1.record(stream)
    e1.synchronize()
    loop_ms = e0.elapsed_time(e1)
    ctx.close()
    icells = int(np.prod(interior))
    value = icells * args.steps / (ms * 1e-3) / 1e9
    loop_value = icells * args.steps / (loop_ms * 1e-3) / 1e9
    line = {
        **base, "impl": "ours", "value": value, "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 1),
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "none", "vs_baseline": None,
        "dtype": "f32", "data": "the reference's TRB set-up (init_trb, physics.hpp), produced by its own program",
        "config": {"workload": "trb_124x124x252_walls_gravity_fp32_central",
                   "configuration_header": "src/cu/ini_files/trb.h", "grid": list(interior), "ghosts": 2,
                   "inputs_vs_L2": "two state buffers of 8.4e7 B each: 1.7e8 B touched per step > L2"},
        "reference_cuda": {"value": ref["gcups"], "ms_per_step": ref["ms_per_step"], "unit": UNIT,
                           "path": "EULERCFD::compute_step (physics.hpp:336-490), the reference's sources "
                                   "built for sm_100a; CUDA events around its calls", "clocks": rclk.summary()},
        "ours_host_loop": {"value": loop_value, "ms_per_step": loop_ms / args.steps,
                           "path": "dg_compute_step(ctx, 1, &dt) per step, dt read back each step, "
                                   "as the reference's loop reads it"},
        "speedup_device": value / ref["gcups"], "speedup_host_loop": loop_value / ref["gcups"],
        "parity_step1": {"rel_l1": errs, "max": max(errs.values()), "dt_rel": abs(dt1 - ref_dt1) / ref_dt1,
                         "region": "interior minus the first layer at each wall"},
        "clocks": clocks, "gpu_launches": step_launches(*interior) * args.steps,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.case == "batch64":
            run_batch(args, world, rank, local)
        elif args.case == "learned":
            run_learned(args, world, rank, local)
        elif args.case == "netfwd":
            run_netfwd(args, world, rank, local)
        elif args.case == "snapshot":
            run_snapshot(args, world, rank, local)
        elif args.case == "corrector":
            run_corrector(args, world, rank, local)
        elif args.case == "refcuda":
            run_refcuda(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
