"""Benchmark of the FDTD (Yee) hot path on B200.

Workload (one bench "step"): the plain-FDTD-with-monitors configuration -- a 256 x 256 x 256
FP32 vacuum grid (Ca = Da = 1, Cb = Db = dt/dx = 0.5), a Gaussian-modulated Jz point source
at the centre (centre period 20 steps, width 10, delay 40), an FP64 running-DFT monitor of Ez
on the plane z = 128 at 8 frequencies over the source band, 1000 time steps from zero fields.
Synthetic inputs with those shapes; fields (1.2 GB) exceed the 126 MB L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: Gcell-updates/s (Nx*Ny*Nz*T / s, boundary cells included, as the reference counts,
gDiamond/gdiamond.hpp:1253).  `value` times the device-resident run (CUDA events on the
launching stream, max over ranks); `e2e` times the same run through the C-ABI with host
buffers: coefficient upload (12 FP32 arrays from pinned memory), reset, 1000 steps, download
of the 6 fields and the monitor sums.  Under torchrun (N ranks) the grid grows to
256 x 256 x 256N and is split into z-slabs, one per rank, with one halo exchange per tiled
launch (--parallelism zslab, the default), or each rank runs its own 256^3 replica
(--parallelism replicas): `scaling` is weak either way.

--impl reference times the reference's own CPU path, gDiamond::update_FDTD_omp, compiled from
the reference sources (oracle/_ref/libgdref.so) on this host's cores, on a bounded number of
time steps of the same 256^3 grid; rank 0 only.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# The reference's OpenMP CPU paths (CPU baseline and reference arm): every host thread, bound
# close; read by the OpenMP runtime when the reference library loads.
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
os.environ.setdefault("OMP_PROC_BIND", "close")


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"

SHAPE = (256, 256, 256)
T_STEPS = 1000
N_FREQS = 8
B_ALG = 96  # algorithmic bytes per FP32 cell-update (6 fields r+w, 12 coefficients r)
WORKLOAD = "fdtd3d_256cube_vacuum_gaussJz_T1000_dft8_zplane"
METRIC = "Gcell-updates/s"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        load = [v for v in sm if mx and v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profile(cfg):
    """DRAM bytes per launch of the tiled kernel from the committed ncu summary (one line per
    configuration), if one of its configurations is the one running now."""
    p = os.path.join(ROOT, "profiles", "fdtd_tiled_256cube_traffic.txt")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        ln = ln.split("#", 1)[0].strip()
        if not ln:
            continue
        kv = dict(part.split("=", 1) for part in ln.split() if "=" in part)
        try:
            if (kv["kernel"] == "fdtd_tiled2") == bool(cfg.get("pairs")) and \
                    (int(kv["width"]), int(kv["blt"]), int(kv["tile_rows"]), int(kv["z_chunks"])) == \
                    (cfg["width"], cfg["blt"], cfg["tile_rows"], cfg["z_chunks"]):
                return float(kv["dram_bytes_per_launch"])
        except (KeyError, ValueError):
            continue
    return None


# ------------------------------------------------------------------ reference arm / CPU


def cpu_reference_sample(target_s=12.0, max_T=400, dt_steps=5):  # dt_steps: a multiple of 5
    """Times the reference's update_FDTD_omp on the 256^3 grid for a bounded number of steps
    (about target_s seconds), and its diamond-tiled update_FDTD_omp_dt(16, 16, 16, 5) for
    dt_steps steps (its schedule is far slower).  Returns a dict: Gcell/s from the wall time
    around the call and from the time the reference prints for its own loop, cores, steps."""
    import oracle
    r = oracle.Reference(*SHAPE)
    r.run_omp(2)
    r.run_omp(4)  # warm (first-touch of the reference's temporaries)
    per_step = max(oracle.Reference.last_printed_seconds() / 4, 1e-4)  # its own loop timer
    T = int(max(2, min(max_T, target_s / per_step)))
    secs = r.run_omp(T)
    printed = oracle.Reference.last_printed_seconds()
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    out = {"omp": {"gcells": n * T / secs / 1e9, "steps": T, "wall_s": secs,
                   "printed_s": printed,
                   "gcells_printed": n * T / printed / 1e9 if printed > 0 else None}}
    try:
        secs_dt = r.run_omp_dt(16, 16, 16, 5, dt_steps)
        printed_dt = oracle.Reference.last_printed_seconds()
        out["omp_dt"] = {"gcells": n * dt_steps / secs_dt / 1e9, "steps": dt_steps,
                         "wall_s": secs_dt, "printed_s": printed_dt, "tiles": [16, 16, 16, 5],
                         "gcells_printed": n * dt_steps / printed_dt / 1e9 if printed_dt > 0
                         else None}
    except Exception as e:  # keep the omp line if the tiled schedule fails
        out["omp_dt"] = {"unavailable": str(e)}
    out["cores"] = oracle.ref().gdref_max_threads()
    r.close()
    return out


def run_reference_arm(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libgdref.so not built"}))
        return 0
    r = oracle.Reference(*SHAPE)
    cores = oracle.ref().gdref_max_threads()
    t2, t4 = r.run_omp(2), r.run_omp(4)
    per_step = max((t4 - t2) / 2, 1e-4)
    T = int(max(2, min(200, 3.0 / per_step)))  # each bench step a ~3 s bounded sample
    for _ in range(args.warmup):
        r.run_omp(T)
    secs, printed = [], []
    for _ in range(args.steps):
        secs.append(r.run_omp(T))
        printed.append(oracle.Reference.last_printed_seconds())
    r.close()
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    total = sum(secs)
    value = n * T * args.steps / total / 1e9
    sample = (f"gDiamond::update_FDTD_omp({T}) on the 256^3 grid (reference constructor "
              f"coefficients and Mz source; same per-cell work as the workload), wall time of "
              f"the call incl. its temporaries and copy-out; {cores} OpenMP threads bound "
              f"close; CPU {cpu_model()}")
    line = {"metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "sample_timesteps": T, "grid": list(SHAPE)},
            "cpu_baseline": {"value": value, "unit": "Gcell-updates/s", "cores": cores,
                             "kind": "reference", "sample": sample, "cpu_model": cpu_model(),
                             "printed_loop_gcells": n * T * args.steps / sum(printed) / 1e9
                             if min(printed) > 0 else None},
            "e2e": {"value": value, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ reference GPU paths


REF_GPU_RUNS = (
    # (binary, driver arguments Tx Ty Tz T, grid, steps): the legal sizes nearest 256^3
    ("gpu_mm_ver2", ("9", "23", "23", "999"), (268, 262, 262), 999),
    ("gpu_mm_ver3", ("20", "52", "52", "1000"), (260, 260, 260), 1000),
)


def _parse_reference_output(text):
    """(label, seconds, Mcells/s) of every timed path in a reference example's stdout: lines
    'gpu runtime (<label>): <s>s' each followed by 'gpu performance: <x>Mcells/s'."""
    import re
    out, label, secs = [], None, None
    for ln in text.splitlines():
        m = re.match(r"gpu runtime \((.*)\): ([0-9.eE+-]+)s", ln.strip())
        if m:
            label, secs = m.group(1), float(m.group(2))
            continue
        m = re.match(r"gpu performance: ([0-9.eE+-]+)\s*Mcells/s", ln.strip())
        if m and label is not None:
            out.append((label, secs, float(m.group(1))))
            label = None
    return out


def reference_gpu_results(timeout=300):
    """The reference's own GPU paths on this GPU: examples/gpu_mm_ver2.cu and gpu_mm_ver3.cu
    compiled unmodified for sm_100a (oracle/_ref, built from the reference sources by
    oracle/Makefile).  Each runs the naive path (update_FDTD_gpu_3D_warp_underutilization_fix)
    and its mix-mapping path at a legal grid size and times them with its own host clock around
    the launch loop (synchronised); the driver then checks the two against each other.  Our
    solver runs the same grid and step count (the reference constructor's coefficients, a
    Gaussian Jz point source at the centre), timed with CUDA events after its autotuning."""
    import torch
    import gdiamond_b200 as gd
    from gdiamond_b200 import workloads as W
    res = {}
    for binary, argv, shape, T in REF_GPU_RUNS:
        path = os.path.join(ROOT, "oracle", "_ref", binary)
        key = f"{binary}_{shape[0]}x{shape[1]}x{shape[2]}_T{T}"
        if not os.path.exists(path):
            res[key] = {"unavailable": f"{path} not built"}
            continue
        try:
            r = subprocess.run([path, *argv], capture_output=True, text=True, timeout=timeout)
            runs = _parse_reference_output(r.stdout)
            entry = {"returncode": r.returncode,
                     "checked_by_driver": "results are matched" in r.stderr,
                     "paths": {lab: {"seconds": sec, "gcells": mc / 1e3} for lab, sec, mc in runs}}
        except subprocess.TimeoutExpired:
            entry = {"unavailable": f"timed out after {timeout} s"}
        # ours, same grid and steps
        nx, ny, nz = shape
        sim = gd.Simulation(nx, ny, nz)
        sim.set_coefficients(W.reference_coefficients(shape))
        sim.set_sources([dict(component="Jz", wave=W.gaussian_wave(T), i=nx // 2, j=ny // 2,
                              k=nz // 2)])
        sim.step(8)  # autotune and warm-up
        sim.reset()
        st = torch.cuda.Stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        sim.step(T, stream=st)
        e1.record(st)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        cfg = sim.config()
        sim.close()
        entry["ours"] = {"seconds": sec, "gcells": nx * ny * nz * T / sec / 1e9,
                         "kernel": cfg}
        for lab, v in entry.get("paths", {}).items():
            entry["ours"][f"speedup_vs_{lab.replace(' ', '_')}"] = v["seconds"] / sec
        res[key] = entry
    return res


# ------------------------------------------------------------------ our arm


def run_ours(args):
    import torch
    import gdiamond_b200 as gd
    from gdiamond_b200 import workloads as W

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if world > 1 and args.parallelism == "zslab":
        return run_zslab(args, rank, world, local, dist, barrier, max_over_ranks)

    shape = tuple(int(v) for v in args.grid.split(","))
    T_run = args.timesteps
    nx, ny, nz = shape
    ncell = nx * ny * nz
    coefs = W.vacuum_coefficients(shape)
    wave = W.gaussian_wave(T_run)
    freqs = W.source_band(N_FREQS)
    src = [dict(component="Jz", wave=wave, i=nx // 2, j=ny // 2, k=nz // 2)]

    sim = gd.Simulation(nx, ny, nz, device=local, kernel=args.kernel, blt=args.blt,
                        tile_rows=args.rows, z_chunks=args.zchunks, min_blocks=args.min_blocks)
    sim.set_coefficients(coefs)
    sim.set_fast_path(not args.no_fast_path)
    if args.cpml:
        # the tiled kernel plus the shell companion (per-step kernels when the grid is small)
        sim.set_cpml(thickness=args.cpml)
    sim.set_sources(src)
    mid = sim.add_dft_monitor("Ez", nz // 2, freqs, scale=1.0)
    stream = torch.cuda.Stream()

    def one_step():
        sim.reset()
        sim.step(T_run, stream=stream)

    # warm-up (the first step also runs the autotuner)
    for _ in range(max(args.warmup, 1)):
        one_step()
    stream.synchronize()
    sim.sync()
    cfg = sim.config()
    sim_fast = sim.fast_path
    launches_per_step = cfg["launches"]

    # ---------------- device-resident timed region
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        sim.reset()
        ev[k][0].record(stream)
        sim.step(T_run, stream=stream)
        ev[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    sim.sync()
    total_ms = max_over_ranks(t_start.elapsed_time(t_end))
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    ms_per_step = total_ms / args.steps
    value = world * ncell * T_run * args.steps / (total_ms / 1e3) / 1e9
    launch_ms = statistics.mean(kern_ms) / launches_per_step

    # ---------------- end to end through the C-ABI with host buffers
    pinned = [torch.empty(ncell, dtype=torch.float32, pin_memory=True).numpy() for _ in range(12)]
    for a in range(12):
        pinned[a][:] = coefs[a]
    fields_out = [torch.empty(ncell, dtype=torch.float32, pin_memory=True).numpy()
                  for _ in range(6)]

    def e2e_step():
        sim.set_coefficients(pinned)
        sim.reset()
        sim.step(T_run)
        for c in range(6):
            sim.get_field(c, out=fields_out[c])
        return sim.get_dft(mid)

    e2e = None
    if not args.no_e2e:
        e2e_step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            re, im = e2e_step()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * ncell * T_run * args.steps / e2e_s / 1e9,
               "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": 12 * ncell * 4 + wave.nbytes,
               "d2h_bytes_per_step": 6 * ncell * 4 + re.nbytes + im.nbytes}

    # ---------------- roofline of the dominant kernel (the tiled kernel)
    hbm, kind = peaks()
    cells_per_launch = ncell * cfg["blt"]
    achieved = B_ALG * cells_per_launch / (launch_ms / 1e3) / 1e9
    traffic = traffic_from_profile(cfg) if shape == SHAPE and not args.cpml else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            r = cpu_reference_sample()
            o = r["omp"]
            cpu = {"value": o["gcells"], "unit": "Gcell-updates/s", "cores": r["cores"],
                   "kind": "reference",
                   "sample": f"gDiamond::update_FDTD_omp({o['steps']}) on the 256^3 grid, "
                             f"{o['wall_s']:.1f} s wall around the call (its printed loop time "
                             f"{o['printed_s']:.2f} s), {r['cores']} OpenMP threads bound close, "
                             f"CPU {cpu_model()} (reference compiled from its sources)",
                   "printed_loop_gcells": o["gcells_printed"], "cpu_model": cpu_model(),
                   "omp_dt": r.get("omp_dt")}
        except Exception as e:  # the reference build may be absent on a user machine
            cpu = {"value": None, "unit": "Gcell-updates/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    sim.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    extra = None
    if world == 1 and not args.no_extras and (shape, T_run) == (SHAPE, T_STEPS):
        extra = {}
        for name, fn in (("mixed", lambda: mixed_results(args)),
                         ("batched", lambda: batched_results(args, ("f16e", "f32"),
                                                             one_at_a_time=False)),
                         ("reference_gpu", reference_gpu_results),
                         ("cpml", cpml_results)):
            try:
                t0 = time.perf_counter()
                extra[name] = fn()
                extra[name]["wall_seconds"] = time.perf_counter() - t0
            except Exception as e:  # an extra configuration must not void the main line
                extra[name] = {"unavailable": f"{type(e).__name__}: {e}"}
    line = {
        "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded shapes of the workload; no dataset)",
        "config": {"workload": (WORKLOAD if (shape, T_run) == (SHAPE, T_STEPS) else
                                f"fdtd3d_{nx}x{ny}x{nz}_vacuum_gaussJz_T{T_run}_dft8_zplane")
                   + (f"_cpml{args.cpml}" if args.cpml else ""),
                   "grid": list(shape), "timesteps": T_run, "cpml_layers": args.cpml,
                   "dft_freqs": N_FREQS, "kernel": cfg["kernel"], "width": cfg.get("width"),
                   "blt": cfg["blt"],
                   "tile_rows": cfg["tile_rows"], "z_chunks": cfg["z_chunks"],
                   "min_blocks": cfg["min_blocks"], "fast_path": sim_fast,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs (1.2 GB of fields) larger than L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "dram_gbs": traffic / (launch_ms / 1e3) / 1e9 if traffic else None,
                     "dram_frac": traffic / (launch_ms / 1e3) / 1e9 / hbm if traffic else None,
                     "dram_bytes_per_cell_update": traffic / cells_per_launch if traffic else None,
                     "note": f"achieved = {B_ALG} B/cell-update x {cells_per_launch} cell-updates "
                             f"per launch / mean launch time {launch_ms:.4f} ms (step time / "
                             f"{launches_per_step} tiled launches; the step's "
                             f"{cfg['dft_folds']} DFT folds included); peak {kind}; "
                             f"temporal tiling lets frac exceed 1; dram_frac = the measured "
                             f"DRAM bytes of one launch (ncu, profiles/) over the same time"},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": (launches_per_step + cfg["dft_folds"]) * args.steps,
        "clocks": clk,
        "extra": extra,
    }
    print(json.dumps(line))
    return 0


def run_zslab(args, rank, world, local, dist, barrier, max_over_ranks):
    """N GPUs advance ONE grid split into z-slabs (gdiamond_b200.slabs.DistZSlab): the workload
    grows with N (256 x 256 x 256N cells, the benchmark's vacuum, Gaussian Jz at the centre of
    the whole grid, 8-frequency DFT of Ez on its middle plane, 1000 steps): weak scaling.  Each
    rank holds its owned planes plus BLT halo planes below and BLT + 1 above; after every
    tiled launch of BLT steps the ranks exchange (2 BLT + 1) planes of all six components per
    interior face with NCCL send/receive into their own device buffers (plain copies, no peer
    loads).  Timed like the single-GPU line: CUDA events on the launching stream, barriers on
    both sides, max over ranks; `value` counts the cells of the whole grid."""
    import torch
    import gdiamond_b200 as gd
    from gdiamond_b200 import workloads as W
    from gdiamond_b200.slabs import DistZSlab

    nx, ny, nz1 = (int(v) for v in args.grid.split(","))
    nz = nz1 * world
    T_run = args.timesteps
    halo = args.blt or 2
    slab = DistZSlab(nx, ny, nz, halo=halo, device=local, tile_rows=args.rows)
    lo, hi = slab.plan.loc[rank]
    own_lo, own_hi = slab.plan.own[rank]
    local_shape = (nx, ny, hi - lo)
    slab.sim.set_coefficients(W.vacuum_coefficients(local_shape))  # vacuum: every slice alike
    wave = W.gaussian_wave(T_run)
    slab.set_sources([dict(component="Jz", wave=wave, i=nx // 2, j=ny // 2, k=nz // 2)])
    slab.add_dft_monitor("Ez", nz // 2, W.source_band(N_FREQS), scale=1.0)
    stream = torch.cuda.Stream(local)  # the timing stream (events); the slab orders after it

    def one_step():
        slab.sim.reset()
        slab.step(T_run, stream)

    for _ in range(max(args.warmup, 1)):
        one_step()
    torch.cuda.synchronize()
    cfg = slab.sim.config()
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        one_step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(e0.elapsed_time(e1))
    ncell = nx * ny * nz
    value = ncell * T_run * args.steps / (total_ms / 1e3) / 1e9
    launch_ms = total_ms / args.steps / max(cfg["launches"], 1)  # exchanges included

    # end to end through the public API with host buffers: each rank uploads its slab's
    # coefficients from pinned memory, steps, and reads back its owned planes (and the monitor)
    e2e = None
    if not args.no_e2e:
        nloc = nx * ny * (hi - lo)
        pinned = [torch.empty(nloc, dtype=torch.float32, pin_memory=True).numpy() for _ in range(12)]
        for a, c in enumerate(W.vacuum_coefficients(local_shape)):
            pinned[a][:] = c
        outs = [torch.empty(nloc, dtype=torch.float32, pin_memory=True).numpy() for _ in range(6)]
        owner, mid = slab.monitors[0]

        def e2e_step():
            slab.sim.set_coefficients(pinned)
            slab.sim.reset()
            slab.step(T_run, stream)
            for c in range(6):
                slab.sim.get_field(c, out=outs[c])
            return slab.sim.get_dft(mid) if owner == rank else (np.zeros(0), np.zeros(0))

        e2e_step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            re, im = e2e_step()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": ncell * T_run * args.steps / e2e_s / 1e9, "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": 12 * nloc * 4 + wave.nbytes,
               "d2h_bytes_per_step": 6 * nloc * 4 + re.nbytes + im.nbytes, "per": "rank"}
    halo_bytes = 0
    for _, _, nk in slab.plan.sends(rank):
        halo_bytes += sum(slab.esz) * nk * nx * ny
    exchanges = (T_run + halo - 1) // halo
    slab.close()
    del slab
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded shapes of the workload; no dataset)",
        "config": {"workload": f"fdtd3d_{nx}x{ny}x{nz}_vacuum_gaussJz_T{T_run}_dft8_zplane",
                   "grid": [nx, ny, nz], "timesteps": T_run, "parallelism": f"zslab{world}",
                   "halo_planes": halo, "kernel": cfg, "gpus_active": world,
                   "halo_bytes_per_exchange_rank0": halo_bytes,
                   "exchanges_per_step": exchanges,
                   "l2": "inputs larger than L2; no flush"},
        "e2e": e2e, "cpu_baseline": None,
        "roofline": {"bound": "hbm", "achieved": B_ALG * nx * ny * (hi - lo) * halo / (launch_ms / 1e3) / 1e9,
                     "peak": peaks()[0], "unit": "GB/s",
                     "frac": B_ALG * nx * ny * (hi - lo) * halo / (launch_ms / 1e3) / 1e9 / peaks()[0],
                     "traffic": None,
                     "note": "rank 0: 96 B/cell-update x local cells x BLT per launch / (step time "
                             "/ launches), halo exchanges included in the time"},
        "gpu_launches": (cfg["launches"] + cfg["dft_folds"]) * args.steps, "clocks": clk,
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ other configurations


def _rel(num, den):
    """sqrt(num / den); a zero reference (a monitor the pulse has not reached) counts as exact
    when the result is zero too, and as an infinite error otherwise."""
    num, den = float(num), float(den)
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return float(np.sqrt(num / den))


def _spectral_error(a, b):
    """Relative L2 error of complex spectra a = (re, im) lists against b."""
    num = sum(np.sum((ar - br) ** 2 + (ai - bi) ** 2) for (ar, ai), (br, bi) in zip(a, b))
    den = sum(np.sum(br ** 2 + bi ** 2) for (br, bi) in b)
    return _rel(num, den)


def _plane_spectrum_error(a, b):
    """Relative L2 error of the plane-integrated spectra S(f) = sum over the monitor plane of
    (re + i im), over all frequencies of the monitors in a (= (re, im) lists) against b."""
    num = den = 0.0
    for (ar, ai), (br, bi) in zip(a, b):
        sa = ar.sum(axis=(1, 2)) + 1j * ai.sum(axis=(1, 2))
        sb = br.sum(axis=(1, 2)) + 1j * bi.sum(axis=(1, 2))
        num += float(np.sum(np.abs(sa - sb) ** 2))
        den += float(np.sum(np.abs(sb) ** 2))
    return _rel(num, den)


def _field_error(F, R):
    num = sum(np.sum((f.astype(np.float64) - r) ** 2) for f, r in zip(F, R))
    den = sum(np.sum(r ** 2) for r in R)
    return float(np.sqrt(num / den))


def _timed(fn, reps=1):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / reps


def fp16_scales(probe, ncell, T, every=2, headroom=2048.0, k_src=None, halfwidth=8):
    """Power-of-two FP16 storage scales from the field peaks of an FP32 run: the largest |value|
    of the E components (and, separately, of the H components) seen every `every` steps of the
    first T steps maps to at most `headroom` (32x below the FP16 maximum, since the field at a
    point source swings between samples and later scattering can focus it; FP16's 2^30 range of
    normal numbers leaves the decayed late-time fields far above its subnormals either way).
    With a point source at plane k_src the peaks are those of the planes within `halfwidth` of
    it (the field is largest at the source), read on the device without copying the grid.  One
    scale per field rather than per component: a component that is zero by symmetry in the
    probe (Hz of a Jz dipole) can grow later by scattering.  Closes `probe`."""
    import torch
    peaks = [0.0] * 6
    nx, ny, nz = probe.shape
    if k_src is None:
        k0, nk = 0, nz
    else:
        k0 = max(0, int(k_src) - halfwidth)
        nk = min(nz, int(k_src) + halfwidth + 1) - k0
    buf = torch.empty(nk * ny * nx, dtype=torch.float32, device="cuda")
    m = torch.zeros(6, dtype=torch.float32, device="cuda")
    for _ in range(0, T, every):
        probe.step(every)
        for c in range(6):
            probe.get_planes_device(c, k0, nk, buf.data_ptr())
            m[c] = torch.maximum(m[c], buf.abs().max())
    torch.cuda.synchronize()
    peaks = [float(v) for v in m.cpu()]
    probe.close()
    e, h = max(peaks[:3]), max(peaks[3:])
    se = float(2.0 ** np.ceil(np.log2(max(e, 1e-30) / headroom)))
    sh = float(2.0 ** np.ceil(np.log2(max(h, 1e-30) / headroom)))
    return [se, se, se, sh, sh, sh]


def run_mixed(args):
    print(json.dumps(mixed_results(args)))
    return 0


def cpml_results(L=10, reps=2):
    """The 256^3 workload (Gaussian Jz at the centre, 8-frequency Ez DFT, 1000 steps) with CPML
    layers of L cells on every face: Gcell-updates/s of the tiled kernel with the shell
    companion and of the per-step CPML kernels (the naive kernel choice), CUDA events on the
    stepping stream, and whether their final fields and DFT sums agree bit for bit."""
    import torch
    import gdiamond_b200 as gd
    from gdiamond_b200 import workloads as W
    nx, ny, nz = SHAPE
    T = T_STEPS
    wave = W.gaussian_wave(T)
    freqs = W.source_band(N_FREQS)
    out, finals = {}, {}
    for name, kernel in (("companion", "auto"), ("per_step", "naive")):
        sim = gd.Simulation(nx, ny, nz, kernel=kernel)
        sim.set_coefficients(W.vacuum_coefficients(SHAPE))
        sim.set_cpml(thickness=L)
        sim.set_sources([dict(component="Jz", wave=wave, i=nx // 2, j=ny // 2, k=nz // 2)])
        mid = sim.add_dft_monitor("Ez", nz // 2, freqs, scale=1.0)
        stream = torch.cuda.Stream()
        sim.step(T, stream=stream)  # tunes (the companion's tiled kernel) outside the timing
        stream.synchronize()
        ms = []
        for _ in range(reps):
            sim.reset()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.step(T, stream=stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        sim.sync()
        cfg = sim.config()
        finals[name] = ([sim.get_field(c) for c in range(6)], sim.get_dft(mid))
        out[name] = {"gcells": nx * ny * nz * T / (min(ms) / 1e3) / 1e9, "ms": ms,
                     "kernel": cfg["kernel"], "blt": cfg["blt"], "tile_rows": cfg["tile_rows"]}
        sim.close()
    (fa, da), (fb, db) = finals["companion"], finals["per_step"]
    same = all(np.array_equal(a.view(np.uint32), b.view(np.uint32)) for a, b in zip(fa, fb))
    same = same and all(np.array_equal(a, b) for a, b in zip(da, db))
    return {"metric": "Gcell-updates/s with CPML layers", "workload": f"{WORKLOAD}_cpml{L}",
            "results": out, "companion_equals_per_step_bitwise": bool(same)}


def mixed_results(args, storages=("f32", "bf16", "f16", "f16e")):
    """Mixed-precision FDTD: 512x512x384 grid, 200 seeded dielectric spheres, Gaussian Jz at the
    centre, FP64 running DFT of Ez at 16 frequencies on the planes z=96 and z=288, 2000 steps.
    FP32, BF16, FP16 and F16E (FP16 E, FP32 H) field storage against an FP64 run of the same
    grid.  FP16 scales come from an FP32 probe of the first 400 steps; its time is reported and
    included in the `gcells_incl_scale_probe` rates."""
    import torch
    import gdiamond_b200 as gd
    from gdiamond_b200 import workloads as W
    shape = tuple(int(v) for v in args.grid.split(",")) if args.grid != "256,256,256" else (512, 512, 384)
    T = args.timesteps if args.timesteps != T_STEPS else 2000
    nx, ny, nz = shape
    eps = W.spheres_eps(shape, n_spheres=200, r_range=(4, 24), eps_range=(1.0, 12.0), seed=0)
    wave = W.gaussian_wave(T)
    freqs = W.source_band(16)
    planes = (nz * 96 // 384, nz * 288 // 384)
    src = [dict(component="Jz", wave=wave, i=nx // 2, j=ny // 2, k=nz // 2)]
    ncell = nx * ny * nz

    def make(storage, scales=None):
        sim = gd.Simulation(nx, ny, nz, storage=storage)
        if scales is not None:
            sim.set_storage_scale(scales)
        sim.set_permittivity(eps)
        sim.set_sources(src)
        for k in planes:
            sim.add_dft_monitor("Ez", k, freqs, scale=1.0)
        return sim

    res = {}
    ref = make("f64")
    t64 = _timed(lambda: ref.step(T) or ref.sync())
    R = [ref.get_field_f64(c) for c in range(6)]
    D64 = [ref.get_dft(m) for m in range(2)]
    nmat = ref.material_count()
    ref.close()
    res["f64"] = {"gcells": ncell * T / t64 / 1e9, "seconds": t64}
    t0 = time.perf_counter()
    f16_scales = fp16_scales(make("f32"), ncell, min(T, 400), k_src=nz // 2)
    t_probe = time.perf_counter() - t0
    t32 = None
    for storage in storages:
        scales = f16_scales if storage in ("f16", "f16e") else None
        sim = make(storage, scales)
        sim.step(2 * 4)  # autotune + warm-up outside the timed run
        sim.reset()
        dt_ = _timed(lambda: sim.step(T) or sim.sync())
        F = [sim.get_field(c) for c in range(6)]
        D = [sim.get_dft(m) for m in range(2)]
        cfg = sim.config()
        sim.close()
        if storage == "f32":
            t32 = dt_
        res[storage] = {"gcells": ncell * T / dt_ / 1e9, "seconds": dt_,
                        "spectral_rel_err_vs_f64": _spectral_error(D, D64),
                        "plane_spectrum_rel_err_vs_f64": _plane_spectrum_error(D, D64),
                        "field_rel_l2_vs_f64": _field_error(F, R),
                        "kernel": cfg, "scales": scales}
        if scales is not None:
            res[storage]["gcells_incl_scale_probe"] = ncell * T / (dt_ + t_probe) / 1e9
        if t32 is not None:
            res[storage]["speedup_vs_f32"] = t32 / dt_
    return {"metric": "Gcell-updates/s and relative error vs FP64", "workload":
            f"fdtd3d_{nx}x{ny}x{nz}_200spheres_gaussJz_T{T}_dft16x2planes",
            "materials": nmat, "fp16_scale_probe_seconds": t_probe, "results": res,
            "data": "synthetic (seeded spheres)"}


def run_batched(args):
    print(json.dumps(batched_results(args, args.batch_storage.split(","))))
    return 0


def batched_results(args, storages, one_at_a_time=True):
    """64 independent uneven simulations (sides from {64,96,128,160,192} per axis, seeded), one
    dielectric slab each, Gaussian Jz at a random interior point, 32-frequency DFT of Ez on one
    plane each, 2000 steps.  Spectra/s of the batched persistent solver (16-bit storage,
    CUDA graph) against the plain FP32 solver run simulation by simulation; spectral error of
    both against FP64 runs."""
    import gdiamond_b200 as gd
    from gdiamond_b200 import workloads as W
    n_sims = args.sims
    T = args.timesteps if args.timesteps != T_STEPS else 2000
    rng = np.random.default_rng(4)
    sides = (64, 96, 128, 160, 192)
    specs = []
    for _ in range(n_sims):
        shape = tuple(int(rng.choice(sides)) for _ in range(3))
        eps = W.slab_eps(shape, rng)
        pos = tuple(int(rng.integers(12, s - 12)) for s in shape)
        specs.append((shape, eps, pos))
    freqs = W.source_band(32)
    wave = W.gaussian_wave(T)
    total_cells = sum(int(np.prod(s[0])) for s in specs)

    def make(spec, storage, scales=None, blt=0):
        shape, eps, pos = spec
        sim = gd.Simulation(*shape, storage=storage, blt=blt)
        if scales is not None:
            sim.set_storage_scale(scales)
        sim.set_permittivity(eps)
        sim.set_sources([dict(component="Jz", wave=wave, i=pos[0], j=pos[1], k=pos[2])])
        sim.add_dft_monitor("Ez", (3 * shape[2]) // 4, freqs, scale=1.0)
        return sim

    def run_each(storage, sync_each=False):
        """Every simulation through the plain (non-batched) solver.  sync_each: one at a time,
        each run finished before the next starts (the reference's GPU calls are synchronous);
        otherwise every handle's asynchronous step call is issued back to back and their
        streams overlap on the GPU."""
        sims = [make(sp, storage) for sp in specs]
        for s in sims:  # autotune each shape outside the timed region
            s.step(4)
            s.reset()
        if sync_each:
            dt_ = _timed(lambda: [s.step(T) or s.sync() for s in sims])
        else:
            dt_ = _timed(lambda: [s.step(T) for s in sims] and [s.sync() for s in sims])
        D = [s.get_dft(0) for s in sims]
        for s in sims:
            s.close()
        return dt_, D

    t64, D64 = run_each("f64")
    t32, D32 = run_each("f32")
    t32s, _ = run_each("f32", sync_each=True) if one_at_a_time else (t32, None)
    out = {"plain_f32_sim_by_sim": {"seconds": t32, "spectra_per_s": n_sims / t32,
                                    "gcells": total_cells * T / t32 / 1e9,
                                    "streams": "overlapped (one stream per handle)",
                                    "spectral_rel_err_vs_f64": float(np.mean(
                                        [_spectral_error([a], [b]) for a, b in zip(D32, D64)]))},
           "plain_f32_one_at_a_time": {"seconds": t32s, "spectra_per_s": n_sims / t32s,
                                       "gcells": total_cells * T / t32s / 1e9},
           "f64_sim_by_sim": {"seconds": t64, "spectra_per_s": n_sims / t64}}
    # FP16 scales valid for every simulation: the fields peak at the source during the pulse
    # and are largest in vacuum (a dielectric lowers Cb), so probe a vacuum copy of the most
    # confined simulation with its source.
    small = min(range(n_sims), key=lambda i: min(specs[i][0]))
    shape0, _, pos0 = specs[small]
    f16 = fp16_scales(make((shape0, np.ones(int(np.prod(shape0)), np.float32), pos0), "f32"),
                      int(np.prod(shape0)), min(T, 300))
    for storage in storages:
        scales = f16 if storage in ("f16", "f16e") else None  # f16e scales E only
        sims = [make(sp, storage, scales, blt=args.blt) for sp in specs]
        batch = gd.Batch(sims)
        batch.step(4)  # batch autotune outside the timed region
        for s in sims:
            s.reset()
        batch.step(T)  # captures the graph
        for s in sims:
            s.reset()

        def one():
            batch.step(T)
            for s in sims:
                s.sync()
        dt_ = _timed(one)
        D = [s.get_dft(0) for s in sims]
        cfg = batch.config()
        errs = [_spectral_error([a], [b]) for a, b in zip(D, D64)]
        perrs = [_plane_spectrum_error([a], [b]) for a, b in zip(D, D64)]
        batch.close()
        for s in sims:
            s.close()
        out[f"batched_{storage}_graph"] = {
            "seconds": dt_, "spectra_per_s": n_sims / dt_, "gcells": total_cells * T / dt_ / 1e9,
            "speedup_vs_plain_f32": t32 / dt_, "speedup_vs_plain_f32_one_at_a_time": t32s / dt_,
            "spectral_rel_err_vs_f64_mean": float(np.mean(errs)),
            "spectral_rel_err_vs_f64_max": float(np.max(errs)),
            "plane_spectrum_rel_err_vs_f64_mean": float(np.mean(perrs)),
            "plane_spectrum_rel_err_vs_f64_max": float(np.max(perrs)), "config": cfg}
    return {"metric": "spectra/s (batched vs plain) at stated spectral error vs FP64",
            "workload": f"{n_sims} uneven sims, sides from {sides}, slab each, T={T}, 32-freq DFT",
            "total_cells": total_cells, "results": out, "data": "synthetic (seeded)"}


def run_surrogate(args):
    """Learned surrogate: 4096 training + 512 held-out designs (a dielectric box in a 96^3
    grid, six numbers each; --train for more), Poynting-flux transmission spectra at 64
    frequencies from the batched FP32 solver (CUDA graph, T=2000; CPML layers on every face,
    or with --boundary pml the reference's graded pseudo-PML); an ensemble of 4 MLPs
    6->256->256->256->64 trained on the GPU (BF16 tensor-core GEMMs, FP32 accumulation, Adam
    lr 1e-3, 200 epochs); held-out spectral error against FDTD with and without the
    ensemble-disagreement fallback, and designs/s of surrogate-with-fallback against the
    batched solver (fallback calls on bucketed, pre-captured batch sizes; three timed runs)."""
    import torch
    from gdiamond_b200 import surrogate as S
    T = args.timesteps if args.timesteps != T_STEPS else S.T_STEPS
    sol = S.SpectrumSolver(T=T, group=256, observable=args.observable, boundary=args.boundary)
    out = {}
    if args.surrogate_data:
        d = np.load(args.surrogate_data)
        train, test = d["train"], d["test"]
        y_train = sol.to_spectra(d["ex_train"], d["flux_train"])
        y_test = sol.to_spectra(d["ex_test"], d["flux_test"])
        sample = test[:256]  # the solver's rate, re-measured on part of the held-out set
        y_s = sol.spectra(sample)  # first call: creates the simulations, tunes, captures
        sol.seconds = 0.0
        sol.spectra(sample)
        out["data"] = {"source": "loaded", "max_rel_diff_vs_loaded":
                       float(S.spectral_error(y_s, y_test[:256]).max())}
        solver_rate = len(sample) / sol.seconds
    else:
        n_active = min(args.active, args.train)
        train = S.sample_designs(args.train - n_active, seed=1)
        test = S.sample_designs(args.test, seed=2)
        t0 = time.perf_counter()
        ex_tr, fl_tr = sol.measure(train)
        if n_active:
            # active sampling within the same budget of solver runs: a first ensemble trained
            # on the random designs picks the designs it is least sure of from a seeded pool
            y0 = sol.to_spectra(ex_tr, fl_tr)
            pilot = S.Surrogate(members=4, seed=7)
            pilot.fit(train, y0, epochs=args.epochs, batch=args.mlp_batch, lr=1e-3, seed=7)
            extra = S.active_designs(pilot, S.sample_designs(8 * args.train, seed=3), n_active)
            pilot.close()
            ex_a, fl_a = sol.measure(extra)
            train = np.concatenate([train, extra])
            ex_tr, fl_tr = np.concatenate([ex_tr, ex_a]), np.concatenate([fl_tr, fl_a])
        t_gen = time.perf_counter() - t0
        sol.seconds = 0.0
        ex_te, fl_te = sol.measure(test)
        solver_rate = len(test) / sol.seconds
        y_train, y_test = sol.to_spectra(ex_tr, fl_tr), sol.to_spectra(ex_te, fl_te)
        out["data"] = {"source": "generated", "train_seconds": t_gen,
                       "active_designs": n_active}
        if args.save_surrogate_data:
            ex0, fl0 = sol.empty()
            np.savez_compressed(args.save_surrogate_data, train=train, test=test,
                                ex_train=ex_tr, flux_train=fl_tr, ex_test=ex_te,
                                flux_test=fl_te, ex_empty=ex0, flux_empty=fl0, freqs=sol.freqs)
    out["batched_solver"] = {"designs_per_s": solver_rate,
                             "config": next(iter(sol.batches.values())).config()}
    out["fallback_buckets"] = "batch sizes padded to powers of two from 4 up to the group"
    sur = S.Surrogate(members=4, seed=0)
    t0 = time.perf_counter()
    losses = sur.fit(train, y_train, epochs=args.epochs, batch=args.mlp_batch, lr=args.mlp_lr,
                     seed=0)
    t_fit = time.perf_counter() - t0
    mean, sd = sur.predict(test)
    err = S.spectral_error(mean, y_test)
    dis = S.Surrogate.disagreement(mean, sd)
    res = {}
    t0 = time.perf_counter()
    sol.warm()  # every bucketed fallback batch size created, tuned and captured once
    t_warm = time.perf_counter() - t0
    for thr in (0.01, 0.02, 0.03, 0.05):
        rates = []
        for _ in range(3):  # three timed evaluations: the run-to-run spread of the rate
            spec, mask, t_s, t_f = sur.evaluate(test, sol, threshold=thr)
            rates.append(len(test) / (t_s + t_f))
        e = S.spectral_error(spec, y_test)
        rate = float(np.median(rates))
        res[f"{thr:g}"] = {"fallback_fraction": float(mask.mean()),
                           "designs_per_s": rate, "designs_per_s_runs": rates,
                           "speedup_vs_batched_solver": rate / solver_rate,
                           "spectral_err_mean": float(e.mean()),
                           "spectral_err_p95": float(np.quantile(e, 0.95)),
                           "spectral_err_max": float(e.max())}
    # the fastest threshold whose mean held-out error stays within 2 %
    ok = [(v["designs_per_s"], k) for k, v in res.items() if v["spectral_err_mean"] <= 0.02]
    best_2pct = None
    if ok:
        r, k = max(ok)
        best_2pct = {"threshold": float(k), "designs_per_s": r,
                     "speedup_vs_batched_solver": res[k]["speedup_vs_batched_solver"],
                     "spectral_err_mean": res[k]["spectral_err_mean"]}
    # inference throughput on device buffers (1M designs), CUDA events on the call's stream
    n_inf = 1 << 20
    x = torch.empty((n_inf, 6), device="cuda").uniform_(-1, 1)
    m_ = torch.empty((n_inf, S.DIMS[-1]), device="cuda")
    s_ = torch.empty_like(m_)
    st = torch.cuda.current_stream()
    for _ in range(3):
        sur.net.predict_device(x.data_ptr(), n_inf, m_.data_ptr(), s_.data_ptr(), st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    reps = 5
    for _ in range(reps):
        sur.net.predict_device(x.data_ptr(), n_inf, m_.data_ptr(), s_.data_ptr(), st)
    e1.record(st)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3 / reps
    dims = S.DIMS
    flop = 2 * sum(a * b for a, b in zip(dims[:-1], dims[1:])) * 4 * n_inf
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    pk = json.load(open(pk_path)) if os.path.exists(pk_path) else {"bf16_tflops": 1590.0}
    out["inference_1M"] = {"designs_per_s": n_inf / sec, "tflops": flop / sec / 1e12,
                           "frac_of_bf16_peak": flop / sec / 1e12 / pk["bf16_tflops"]}
    out["surrogate"] = {"observable": args.observable, "boundary": args.boundary,
                        "adam_lr": args.mlp_lr,
                        "flux_plane": sol.monitor_k, "train_seconds": t_fit,
                        "bucket_warmup_seconds": t_warm,
                        "epochs": args.epochs, "batch": args.mlp_batch,
                        "final_loss_per_member": [float(v) for v in losses[-1]],
                        "heldout_err_mean_no_fallback": float(err.mean()),
                        "heldout_err_median_no_fallback": float(np.median(err)),
                        "heldout_err_p95_no_fallback": float(np.quantile(err, 0.95)),
                        "baseline_mean_spectrum_err": float(S.spectral_error(
                            np.broadcast_to(y_train.mean(0), y_test.shape), y_test).mean()),
                        "disagreement_median": float(np.median(dis)),
                        "with_fallback": res, "fastest_within_2pct_err": best_2pct}
    sur.close()
    sol.close()
    line = {"metric": "designs/s (surrogate with FDTD fallback vs batched solver) at stated "
                      "held-out spectral error",
            "workload": f"box designs in 96^3, T={T}, 64-freq transmission ({args.observable}, "
                        f"{'CPML' if args.boundary == 'cpml' else 'graded pseudo-PML'}), "
                        f"{len(train)} train + {len(test)} held-out",
            "results": out, "data": "synthetic (seeded designs)"}
    print(json.dumps(line))
    return 0


def run_mlp(args):
    """The surrogate's tensor-core GEMMs alone: ensemble inference (4 members, 6->256->256->256
    ->64, BF16 operands, FP32 accumulation) on `--designs` synthetic designs resident in HBM,
    timed with CUDA events on the call's stream, and training throughput (forward + backward +
    Adam, minibatches of 64) on 4096 synthetic designs; both GEMM paths."""
    import torch
    import gdiamond_b200 as gd
    from gdiamond_b200 import surrogate as S
    dims, E, n = S.DIMS, 4, args.designs
    flop_fwd = 2 * sum(a * b for a, b in zip(dims[:-1], dims[1:])) * E
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    pk = json.load(open(pk_path)) if os.path.exists(pk_path) else {"bf16_tflops": 1590.0}
    peak, peak_kind = float(pk["bf16_tflops"]), "measured" if "hbm_gbs" in pk else "fallback"
    x = torch.empty((n, dims[0]), device="cuda").uniform_(-1, 1)
    mean = torch.empty((n, dims[-1]), device="cuda")
    sd = torch.empty_like(mean)
    rng = np.random.default_rng(0)
    xs = rng.uniform(-1, 1, (4096, dims[0])).astype(np.float32)
    ys = rng.normal(0, 1, (4096, dims[-1])).astype(np.float32)
    out = {}
    st = torch.cuda.current_stream()
    for gemm in ("auto", "tcgen05", "mma_sync"):
        net = gd.MLP(dims, members=E, seed=0, gemm=gemm)
        for _ in range(args.warmup):
            net.predict_device(x.data_ptr(), n, mean.data_ptr(), sd.data_ptr(), st)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            net.predict_device(x.data_ptr(), n, mean.data_ptr(), sd.data_ptr(), st)
        e1.record(st)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / args.steps
        net.set_data(xs, ys)
        net.train(epochs=1, batch=64)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        net.train(epochs=args.train_epochs, batch=64)
        t_train = time.perf_counter() - t0
        out[gemm] = {"inference_designs_per_s": n / sec, "inference_ms": sec * 1e3,
                     "inference_tflops": flop_fwd * n / sec / 1e12,
                     "frac_of_bf16_peak": flop_fwd * n / sec / 1e12 / peak,
                     "train_epochs_per_s": args.train_epochs / t_train,
                     "train_designs_per_s": args.train_epochs * len(xs) / t_train}
        net.close()
    line = {"metric": "MLP ensemble inference TFLOP/s (BF16 tensor cores, FP32 accumulate)",
            "workload": f"4-member ensemble {dims}, {n} designs per call; training minibatches "
                        f"of 64 on 4096 designs",
            "peak_bf16_tflops": peak, "peak_kind": peak_kind, "results": out,
            "data": "synthetic"}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer run")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision, batched and reference-GPU lines that the "
                         "default run adds under 'extra'")
    ap.add_argument("--grid", default="256,256,256", help="NX,NY,NZ (profiling cases)")
    ap.add_argument("--timesteps", type=int, default=T_STEPS)
    ap.add_argument("--kernel", default="auto",
                    choices=["auto", "naive", "tiled", "tiled_w32", "tiled_w64", "tiled_w32p"])
    ap.add_argument("--blt", type=int, default=0, help="force time steps per launch")
    ap.add_argument("--rows", type=int, default=0, help="force tile rows")
    ap.add_argument("--zchunks", type=int, default=0, help="force z-chunks")
    ap.add_argument("--min-blocks", type=int, default=0, help="force the register cap")
    ap.add_argument("--parallelism", default="zslab", choices=["zslab", "replicas"],
                    help="N > 1: one grid split into z-slabs over the GPUs (halo exchange), or "
                         "an independent replica per GPU")
    ap.add_argument("--cpml", type=int, default=0,
                    help="CPML layers of this many cells on every face (the per-step E/H "
                         "kernels instead of the tiled kernel)")
    ap.add_argument("--no-fast-path", action="store_true",
                    help="force the general per-cell path of the x-pair kernels")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "mixed", "batched", "surrogate", "mlp"],
                    help="plain: the benchmark line; mixed / batched: the precision and "
                         "batching configurations (separate JSON lines)")
    ap.add_argument("--sims", type=int, default=64, help="batched workload: simulations")
    ap.add_argument("--batch-storage", default="bf16,f16,f16e,f32",
                    help="batched workload: storages of the batched runs")
    ap.add_argument("--designs", type=int, default=1 << 20, help="mlp: designs per inference")
    ap.add_argument("--train-epochs", type=int, default=10, help="mlp: timed training epochs")
    ap.add_argument("--train", type=int, default=4096,
                    help="surrogate: training designs (4096 as the configuration states)")
    ap.add_argument("--test", type=int, default=512, help="surrogate: held-out designs")
    ap.add_argument("--active", type=int, default=1024,
                    help="surrogate: of the training designs, this many chosen by the "
                         "disagreement of a first ensemble (active sampling)")
    ap.add_argument("--epochs", type=int, default=200, help="surrogate: training epochs")
    ap.add_argument("--mlp-batch", type=int, default=64, help="surrogate: minibatch rows")
    ap.add_argument("--mlp-lr", type=float, default=1e-3,
                    help="surrogate: Adam learning rate of the ensemble (the config's 1e-3)")
    ap.add_argument("--boundary", default="cpml", choices=["pml", "cpml"],
                    help="surrogate: CPML layers on every face (default) or the reference's "
                         "graded pseudo-PML")
    ap.add_argument("--observable", default="flux", choices=["flux", "amplitude"],
                    help="surrogate: transmission observable")
    ap.add_argument("--surrogate-data", default="",
                    help="surrogate: .npz of designs and measurements from an earlier run")
    ap.add_argument("--save-surrogate-data", default="",
                    help="surrogate: write the generated designs and measurements (.npz)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "surrogate":
        return run_surrogate(args)
    if args.workload == "mlp":
        return run_mlp(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
