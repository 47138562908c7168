"""PSTM throughput benchmark (pairs of output sample x input trace per second).

Default workload: the 3D PSTM, plain FP32 -- 500k traces x 1000 samples at 4 ms,
midpoints uniform over 5 x 5 km, offsets uniform 0-3000 m, azimuths uniform,
200 Ricker-30 Hz diffractors + 3 % noise, V_rms(t0, x, y) rising 1500 -> 3500
m/s with a +-5 % lateral sinusoid, output 200 x 200 x 1000 at 25 m, 1000 m
aperture, 60 deg angle.  Synthetic, seeded.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f32|bf16|f16]
                  [--antialias] [--utm]
  python bench.py --impl reference ...   (CPU port of the reference kernel)
  python bench.py --config batched | lsq | velocity | time_rms

``--antialias --utm --storage bf16|f16`` is the anti-aliased workload with
traces stored in 16 bits and world coordinates offset by a UTM origin.  Every
run quotes ``error_vs_fp64``: the rel-L2 of its image against the FP64 oracle on
64 columns spread over the grid (2 x 2 clusters at the corners, the edge
midpoints, the centre and seeded interior positions; ``--err-clusters``), and
the fold mismatch as a fraction of the pairs checked.

One JSON line on rank 0.  ``value`` = pairs / device time of one step with the
inputs resident in HBM (stage traces, then forward migration with the fold; the geometry
plan is built once, outside the timed region), max over ranks; ``e2e`` = the same
metric through MigrationEngine.migrate_bin_full with pinned host inputs,
host<->device copies and plan construction inside the timed region.
Inputs (2 GB of traces) are larger than the 126 MB L2, so no L2 flush is needed.
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
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MUFU_PER_SM_CLK = 16
RSQRT_PER_PAIR = 2
# DRAM bytes per trace-list entry of the forward gather, from the ncu capture
# of the 100k-trace case (31.2 GB / 9.0 M entries, 16-column tiles, expanded float32 rows);
# the traffic of a full launch is scaled by its list entries.
DRAM_BYTES_PER_LIST_ENTRY = 3470.0


def peaks():
    p = {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "source": "fallback"}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        p.update(hbm_gbs=float(m["hbm_gbs"]), sm_max_mhz=float(m.get("sm_max_mhz", 1965.0)),
                 source="measured")
    except Exception:
        pass
    return p


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        try:
            p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                  "--format=csv,noheader,nounits", "-lms", "200"],
                                 stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        while not self._stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            self.rows.append([x.strip() for x in line.split(",")])
        p.terminate()
        try:
            p.wait(timeout=5)
        except Exception:
            p.kill()

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        time.sleep(0.3)
        self._stop.set()
        self._t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


UTM_ORIGIN = (5.0e5, 6.0e6)


def make_workload(device, rank: int, args):
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=args.traces, seed=2025 + rank, device=device,
                               n_samples=args.samples, n_il=args.grid, n_xl=args.grid,
                               utm_origin=UTM_ORIGIN if getattr(args, "utm", False) else (0.0, 0.0))


def workload_name(args) -> str:
    if (args.storage == "f32" and args.traces == 500_000 and not args.antialias
            and not args.utm and args.samples == 1000 and args.grid == 200):
        return ("3D PSTM plain FP32 (500k traces x 1000 samples, 200x200x1000 output, "
                "V_rms(t0,x,y), A=1000 m, 60 deg)")
    extra = []
    if args.antialias:
        extra.append(f"triangle anti-alias (half-width <= {args.aa_lmax:g} samples)")
    if args.utm:
        extra.append(f"UTM origin ({UTM_ORIGIN[0]:.0e}, {UTM_ORIGIN[1]:.0e}) m")
    return (f"3D PSTM {args.storage} storage{', ' if extra else ''}{', '.join(extra)} "
            f"({args.traces} traces x {args.samples} samples, {args.grid}x{args.grid}x"
            f"{args.samples} output, V_rms(t0,x,y), A=1000 m, 60 deg)")


def crop_traces(s, cols):
    """Traces with both legs inside the aperture of some column of the crop."""
    il = cols // s.n_xl
    xl = cols % s.n_xl
    cx = s.origin_x + il * s.il_spacing
    cy = s.origin_y + xl * s.xl_spacing
    mx, my = cx.mean(), cy.mean()
    r = s.max_aperture_m + float(np.hypot(cx - mx, cy - my).max()) + 1.0
    keep = ((np.hypot(s.source_x - mx, s.source_y - my) <= r)
            & (np.hypot(s.receiver_x - mx, s.receiver_y - my) <= r))
    return np.nonzero(keep)[0], cx, cy


def run_fp64_crop(s, cols, antialias: bool, l_max: float):
    """FP64 oracle image of the crop columns (checker and, for the anti-alias
    workload, the CPU baseline: the reference has no anti-aliased migration)."""
    from oracle import pstm_fp64 as O
    idx, cx, cy = crop_traces(s, cols)
    tr = s.traces[:, torch.from_numpy(idx).to(s.traces.device)].cpu().numpy()
    n_t = s.n_times
    t_ms = (np.arange(n_t, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    vel = s.vrms.reshape(n_t, -1)[:, cols]
    ox, oy = s.origin_x, s.origin_y
    t0 = time.perf_counter()
    img, fold = O.migrate_fp64(tr, s.source_x[idx] - ox, s.source_y[idx] - oy,
                               s.receiver_x[idx] - ox, s.receiver_y[idx] - oy, cx - ox, cy - oy,
                               t_ms, vel, s.dt_ms, 0.0, s.max_aperture_m, s.max_angle_deg,
                               antialias=antialias, dx_out=s.il_spacing, dy_out=s.xl_spacing,
                               l_max=l_max)
    return img, fold, time.perf_counter() - t0, int(idx.size)


def cpu_crop_columns(s, side: int):
    """Flat column indices of a centred side x side crop of the output grid."""
    i0 = s.n_il // 2 - side // 2
    j0 = s.n_xl // 2 - side // 2
    il = np.arange(i0, i0 + side)[:, None]
    xl = np.arange(j0, j0 + side)[None, :]
    return np.sort((il * s.n_xl + xl).ravel())


def error_clusters(n_il: int, n_xl: int, n_clusters: int = 16, seed: int = 11):
    """2 x 2 column clusters checked against the FP64 oracle: the four corners,
    the four edge midpoints, the centre, and seeded random interior clusters
    (16 clusters = 64 columns by default).  Returns a list of flat column
    index arrays (il * n_xl + xl)."""
    a_il, a_xl = max(n_il - 2, 0), max(n_xl - 2, 0)
    anchors = [(0, 0), (0, a_xl), (a_il, 0), (a_il, a_xl),
               (0, a_xl // 2), (a_il // 2, 0), (a_il, a_xl // 2), (a_il // 2, a_xl),
               (a_il // 2, a_xl // 2)]
    rs = np.random.RandomState(seed)
    while len(anchors) < n_clusters:
        anchors.append((int(rs.randint(1, max(a_il, 2))), int(rs.randint(1, max(a_xl, 2)))))
    out = []
    for i0, j0 in anchors[:n_clusters]:
        il = np.arange(i0, min(i0 + 2, n_il))[:, None]
        xl = np.arange(j0, min(j0 + 2, n_xl))[None, :]
        out.append(np.sort((il * n_xl + xl).ravel()))
    return out


def fp64_check(s, img_cols, fold_cols, clusters, antialias: bool, l_max: float, storage: str,
               threads: int = 0):
    """rel-L2 of the image columns against the FP64 oracle over all clusters
    (one oracle run per cluster with the traces in its aperture, in a thread
    pool), and the fold mismatch as a count and a fraction of the pairs."""
    import concurrent.futures as cf
    dev = img_cols.device
    todo = []
    for cols in clusters:
        e = torch.from_numpy(cols).to(dev)
        todo.append((cols, img_cols[:, e].double().cpu().numpy(),
                     fold_cols[:, e].double().cpu().numpy()))
    n_thr = threads or min(len(todo), max(1, len(os.sched_getaffinity(0))))
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=n_thr) as ex:
        res = list(ex.map(lambda c: run_fp64_crop(s, c[0], antialias, l_max), todo))
    wall = time.perf_counter() - t0
    num = den = mism = pairs = 0.0
    worst = 0.0
    n_tr = 0
    for (cols, gi, gf), (oi, of, _, ntr) in zip(todo, res):
        num += float(np.sum((gi - oi) ** 2))
        d = float(np.sum(oi ** 2))
        den += d
        worst = max(worst, float(np.linalg.norm(gi - oi) / max(np.sqrt(d), 1e-300)))
        mism += float(np.abs(gf - of).sum())
        pairs += float(of.sum())
        n_tr += ntr
    return {"rel_l2": float(np.sqrt(num / max(den, 1e-300))), "worst_cluster_rel_l2": worst,
            "fold_mismatch": mism, "fold_mismatch_frac": mism / max(pairs, 1.0),
            "pairs_checked": pairs, "columns": int(sum(c.size for c in clusters)),
            "clusters": "2x2 columns at the 4 corners, 4 edge midpoints, the centre and "
                        f"{max(len(clusters) - 9, 0)} seeded interior positions",
            "traces_in_apertures": n_tr, "oracle_wall_s": wall, "oracle_threads": n_thr,
            "oracle": "FP64 restatement" + (" with anti-alias" if antialias else ""),
            "storage": storage, "sum_sq_err": num, "sum_sq_ref": den}


def merge_checks(checks, storage: str):
    """One error summary over several fp64_check results (e.g. several classes)."""
    num = sum(c["sum_sq_err"] for c in checks)
    den = sum(c["sum_sq_ref"] for c in checks)
    mism = sum(c["fold_mismatch"] for c in checks)
    pairs = sum(c["pairs_checked"] for c in checks)
    return {"rel_l2": float(np.sqrt(num / max(den, 1e-300))),
            "worst_cluster_rel_l2": max(c["worst_cluster_rel_l2"] for c in checks),
            "fold_mismatch": mism, "fold_mismatch_frac": mism / max(pairs, 1.0),
            "pairs_checked": pairs, "columns": sum(c["columns"] for c in checks),
            "oracle_wall_s": sum(c["oracle_wall_s"] for c in checks),
            "oracle": checks[0]["oracle"], "storage": storage}


def run_cpu_port(s, cols, fold_pairs_cols):
    """Reference-port CPU timing on a column crop (all traces supplied)."""
    from oracle.ref_port import engine_full_port
    threads = len(os.sched_getaffinity(0))
    torch.set_num_threads(threads)
    tr = s.traces.cpu().numpy()
    t0 = time.perf_counter()
    engine_full_port(tr, s.source_x - s.origin_x, s.source_y - s.origin_y,
                     s.receiver_x - s.origin_x, s.receiver_y - s.origin_y, 0.0, 0.0,
                     s.il_spacing, s.xl_spacing, s.n_il, s.n_xl, s.dt_ms, 0.0, s.n_times,
                     float(s.vrms.mean()), s.max_aperture_m, s.max_angle_deg,
                     column_subset=cols)
    el = time.perf_counter() - t0
    return {"value": fold_pairs_cols / el / 1e9, "unit": "Gpairs/s", "cores": threads,
            "kind": "port", "seconds": el,
            "sample": f"centred {int(round(len(cols) ** 0.5))}x{int(round(len(cols) ** 0.5))}-column "
                      f"crop x {s.n_times} samples, all {s.n_traces} traces supplied, "
                      f"{fold_pairs_cols:.3e} pairs; constant V = mean V_rms"}


def bench_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.antialias:
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference migrators have no anti-alias filter on this path"}),
              flush=True)
        return
    s = make_workload("cpu" if not torch.cuda.is_available() else "cuda", 0, args)
    from oracle import pstm_fp64 as O
    cols = cpu_crop_columns(s, args.crop)
    il = cols // s.n_xl
    xl = cols % s.n_xl
    cx = s.origin_x + il * s.il_spacing
    cy = s.origin_y + xl * s.xl_spacing
    t_ms = (np.arange(s.n_times, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    pairs = O.count_pairs_fp64(s.source_x, s.source_y, s.receiver_x, s.receiver_y, cx, cy, t_ms,
                               float(s.vrms.mean()), s.max_aperture_m, s.max_angle_deg)
    vals = []
    for i in range(args.warmup + args.steps):
        r = run_cpu_port(s, cols, pairs)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median([r["value"] for r in vals])
    ms = statistics.median([r["seconds"] for r in vals]) * 1e3
    cb = dict(vals[0])
    cb["value"] = v
    cb.pop("seconds", None)
    print(json.dumps({
        "metric": "PSTM Gpairs/s (out-sample x trace)", "value": v, "unit": "Gpairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": workload_name(args), "storage": "f32",
                   "traces": s.n_traces, "samples": s.n_samples},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "Gpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def bench_ours(args):
    import torch.distributed as dist
    from seisproc_b200 import _lib
    from seisproc_b200.kirchhoff import PSTMPlan
    from seisproc_b200.engine import MigrationEngine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    L = _lib.lib()

    t_gen = time.perf_counter()
    s = make_workload(dev, rank, args)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    n_t = s.n_times
    vel = torch.from_numpy(s.vrms.reshape(n_t, -1)).to(dev)
    coords = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
              for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan_kw = dict(n_il=s.n_il, n_xl=s.n_xl, n_times=n_t, origin_x=s.origin_x,
                   origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                   xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                   in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                   max_angle_deg=s.max_angle_deg, storage=args.storage,
                   antialias=args.antialias, aa_dx=s.il_spacing, aa_dy=s.xl_spacing,
                   aa_max_halfwidth=args.aa_lmax, forward_only=True)
    torch.cuda.synchronize()
    t_tune = time.perf_counter()
    variant = args.variant
    if variant == "auto":
        from seisproc_b200 import autotune
        variant = autotune.choose_variant(coords, velocity=vel, **plan_kw)
    t_tune = time.perf_counter() - t_tune
    t_plan = time.perf_counter()
    plan = PSTMPlan(*coords, variant=variant, **plan_kw)
    torch.cuda.synchronize()
    t_plan = time.perf_counter() - t_plan
    traces = s.traces
    image = torch.empty((n_t, s.n_il, s.n_xl), device=dev)
    fold = torch.empty_like(image)

    def step(ev=None):
        if ev:
            ev[0].record()
        plan.load_traces(traces)
        if ev:
            ev[1].record()
        plan.migrate_loaded(vel, image=image, fold=fold)  # fold counted in the same launch
        if ev:
            ev[2].record()
        return fold

    for _ in range(args.warmup):
        f = step()
    plan.check()
    pairs = float(f.double().sum().item())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    l0 = L.pstm_launch_count()
    with ClockSampler(local) as clk:
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        for i in range(args.steps):
            step(evs[i])
        end.record()
        torch.cuda.synchronize()
    launches = L.pstm_launch_count() - l0
    plan.check()
    total_ms = start.elapsed_time(end)
    stage_ms = [e[0].elapsed_time(e[1]) for e in evs]
    fwd_ms = [e[1].elapsed_time(e[2]) for e in evs]
    t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tp = torch.tensor([pairs], device=dev, dtype=torch.float64)
        dist.all_reduce(tp)
        pairs_all = float(tp.item())
    else:
        pairs_all = pairs
    total_ms = float(t.item())
    ms_step = total_ms / args.steps
    value = pairs_all * args.steps / (total_ms * 1e-3) / 1e9

    # e2e through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host_tr = torch.empty(traces.shape, dtype=torch.float32, pin_memory=True)
        host_tr.copy_(traces)
        host_v = torch.empty(s.vrms.shape, dtype=torch.float32, pin_memory=True)
        host_v.copy_(torch.from_numpy(s.vrms))
        host_c = []
        for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y):
            h = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            h.copy_(torch.from_numpy(a))
            host_c.append(h)
        eng = MigrationEngine(storage=args.storage, variant=args.variant)
        kw = dict(origin_x=s.origin_x, origin_y=s.origin_y, il_spacing=s.il_spacing,
                  xl_spacing=s.xl_spacing, azimuth_deg=0.0, n_il=s.n_il, n_xl=s.n_xl,
                  dt_ms=s.dt_ms, t_min_ms=0.0, n_times=n_t, max_aperture_m=s.max_aperture_m,
                  max_angle_deg=s.max_angle_deg, normalize=True, antialias=args.antialias,
                  aa_max_halfwidth=args.aa_lmax)
        run = lambda: eng.migrate_bin_full(host_tr.numpy(), *[h.numpy() for h in host_c],
                                           velocity_model=host_v.numpy(), **kw)
        run()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        # each call timed between CUDA events on the stream (the call returns
        # numpy arrays, so it ends synchronised); the median call is reported
        e_steps = max(3, min(args.steps, 5))
        calls = []
        for _ in range(e_steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            img_np, fold_np = run()
            b.record()
            torch.cuda.synchronize()
            calls.append(a.elapsed_time(b))
        te = torch.tensor([statistics.median(calls)], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e_ms = float(te.item())
        h2d = host_tr.numel() * 4 + sum(h.numel() * 8 for h in host_c) + host_v.numel() * 4
        d2h = img_np.nbytes + fold_np.nbytes
        e2e = {"value": pairs_all / (e_ms * 1e-3) / 1e9, "unit": "Gpairs/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e_ms, "ms_calls": [round(c, 1) for c in calls],
               "statistic": "median call"}
        # the reference worker's calling pattern: a bin's traces come from a
        # reader as (n_traces, n_samples) pageable arrays; streamed here through
        # page-locked chunks into trace-major staging (no host transpose)
        if world == 1:
            from seisproc_b200.ingest import NumpyDataReader
            reader = NumpyDataReader(np.ascontiguousarray(host_tr.numpy().T))
            idx = np.arange(reader.n_traces)
            c_np = [h.numpy() for h in host_c]
            run_r = lambda: eng.migrate_bin_from_reader(reader, idx, *c_np,
                                                        velocity_model=host_v.numpy(), **kw)
            run_r()
            rc = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                run_r()
                rc.append((time.perf_counter() - t0) * 1e3)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.migrate_bin_full(reader.read_traces(idx).T, *c_np,
                                 velocity_model=host_v.numpy(), **kw)
            ref_ms = (time.perf_counter() - t0) * 1e3
            r_ms = statistics.median(rc)
            e2e["reader"] = {
                "value": pairs_all / (r_ms * 1e-3) / 1e9, "unit": "Gpairs/s", "ms_per_step": r_ms,
                "ms_calls": [round(c, 1) for c in rc],
                "source": "NumpyDataReader over a pageable (n_traces, n_samples) array",
                "reference_pattern_ms": ref_ms,
                "reference_pattern": "read_traces(idx).T then migrate_bin_full (host transpose "
                                     "and pageable upload), one call"}
            del reader

    result = None
    if rank == 0:
        pk = peaks()
        clocks = clk.summary()
        fwd_avg = statistics.mean(fwd_ms)
        mufu_per_pair = RSQRT_PER_PAIR + (1 if args.antialias else 0)
        peak_pairs = 148 * MUFU_PER_SM_CLK / mufu_per_pair * pk["sm_max_mhz"] * 1e6 / 1e12
        achieved = pairs / (fwd_avg * 1e-3) / 1e12
        plain_f32 = args.storage == "f32" and not args.antialias
        traffic = DRAM_BYTES_PER_LIST_ENTRY * plan.stats()["list_entries"] if plain_f32 else None
        roof = {"bound": "mufu", "achieved": achieved, "peak": peak_pairs, "unit": "Tpairs/s",
                "frac": achieved / peak_pairs, "traffic": traffic,
                "mufu_per_pair": mufu_per_pair,
                "traffic_note": "DRAM bytes per launch scaled from the ncu capture of the "
                                "100k-trace case by list entries" if plain_f32 else
                                "not captured for this storage/filter",
                "hbm_achieved_gbs": traffic / (fwd_avg * 1e-3) / 1e9 if traffic else None,
                "hbm_peak_gbs": pk["hbm_gbs"],
                "peak_source": f"{pk['source']} sm_max_mhz {pk['sm_max_mhz']}",
                "kernel": "pstm_gather2_kernel (forward, fold counted in the same launch)",
                "kernel_ms": fwd_avg, "stage_ms": statistics.mean(stage_ms)}
        cb = None
        err = None
        if world == 1 and not args.no_cpu:
            img_cols = image.reshape(n_t, -1)
            fold_cols_t = f.reshape(n_t, -1)
            # error of this result against the FP64 oracle on columns spread over the grid
            err = fp64_check(s, img_cols, fold_cols_t,
                             error_clusters(s.n_il, s.n_xl, args.err_clusters),
                             args.antialias, args.aa_lmax, args.storage)
            if args.antialias:
                # the reference has no anti-aliased migration: the FP64 oracle
                # on a centred crop is the CPU baseline
                ecols = cpu_crop_columns(s, args.err_crop)
                eidx = torch.from_numpy(ecols).to(dev)
                oi, of, o_sec, o_tr = run_fp64_crop(s, ecols, args.antialias, args.aa_lmax)
                gf = fold_cols_t[:, eidx].double().cpu().numpy()
                pc = float(gf.sum())
                cb = {"value": pc / o_sec / 1e9, "unit": "Gpairs/s", "cores": 1, "kind": "port",
                      "sample": f"centred {args.err_crop}x{args.err_crop}-column crop x {n_t} "
                                f"samples, {o_tr} traces in its aperture, {pc:.3e} pairs; FP64 "
                                "numpy restatement with anti-alias (the reference has none)"}
            else:
                cols = cpu_crop_columns(s, args.crop)
                fold_cols = float(fold_cols_t[:, torch.from_numpy(cols).to(dev)].double().sum())
                cb = run_cpu_port(s, cols, fold_cols)
                cb.pop("seconds", None)
                # the whole workload at the crop's rate (extrapolated, not run)
                cb["full_workload_s_extrapolated"] = pairs_all / (cb["value"] * 1e9)
        result = {
            "metric": "PSTM Gpairs/s (out-sample x trace)", "value": value, "unit": "Gpairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args), "storage": args.storage,
                       "antialias": bool(args.antialias),
                       "traces_per_gpu": s.n_traces, "pairs_per_step_per_gpu": pairs,
                       "plan": plan.stats(), "plan_build_s": t_plan, "datagen_s": t_gen,
                       "shape_choice": ("autotuner (cached per problem class; this run's "
                                        f"choice took {t_tune:.2f} s)"
                                        if args.variant == "auto" else "fixed --variant"),
                       "l2": "inputs (traces) larger than L2; no flush",
                       "parallelism": (f"replicas: one independent survey per rank, {world} rank(s), "
                                       "no collective") if world > 1 else "one GPU"},
            "roofline": roof, "cpu_baseline": cb, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clocks, "error_vs_fp64": err,
        }
        print(json.dumps(result), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def batched_surveys(args, dev):
    """The batched workload: the first ``args.classes`` of 64 offset/azimuth
    classes (8 offset bins x 8 azimuth sectors, trace counts log-uniform
    2k-40k, seed 64), one synthetic survey per class sharing diffractors,
    velocity and grid."""
    from seisproc_b200 import synthetic
    counts = synthetic.class_counts_loguniform(64, 2000, 40000, seed=64)[:args.classes]
    return synthetic.survey_classes(counts, seed=64, device=dev, n_samples=args.samples,
                                    n_il=args.grid, n_xl=args.grid)


def class_plans(surveys, storage: str, variant, dev, vel):
    """One forward_only plan per class; ``variant="auto"`` takes each class's
    kernel shape from the autotuner (cached per problem class)."""
    from seisproc_b200 import autotune
    from seisproc_b200.kirchhoff import PSTMPlan
    plans = []
    for s in surveys:
        c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
             for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
        kw = dict(n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                  origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                  xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                  in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                  max_angle_deg=s.max_angle_deg, storage=storage, forward_only=True)
        v = autotune.choose_variant(c, velocity=vel, **kw) if variant == "auto" else variant
        plans.append(PSTMPlan(*c, variant=v, **kw))
    return plans


def checked_classes(pairs_per_class, n: int = 8, seed: int = 8):
    """Classes checked against the FP64 oracle: the four with the most pairs and
    seeded others among those with pairs."""
    live = [i for i, p in enumerate(pairs_per_class) if p > 0]
    top = sorted(live, key=lambda i: -pairs_per_class[i])[:4]
    rest = [i for i in live if i not in top]
    rs = np.random.RandomState(seed)
    extra = list(rs.choice(rest, size=min(n - len(top), len(rest)), replace=False)) if rest else []
    return sorted(top + [int(i) for i in extra])


def shard_partition(s, world: int):
    """The sharded mode's partition of one survey: inline slabs (sizes
    differing by at most one) and, per slab, the traces whose two legs reach
    it within the aperture (its halo)."""
    from seisproc_b200 import sharding as S
    slabs = S.inline_slabs(s.n_il, world)
    halos = []
    for il0, il1 in slabs:
        box = S.slab_bbox(s.origin_x, s.origin_y, s.il_spacing, 0.0, 0.0, s.xl_spacing, s.n_xl,
                          il0, il1)
        halos.append(S.halo_traces(s.source_x, s.source_y, s.receiver_x, s.receiver_y, box,
                                   s.max_aperture_m))
    return slabs, halos


def shard_aggregate(ms: float, pairs: float, device, group=None):
    """Whole-job figures from one rank's timed milliseconds and pairs: the
    slowest rank's time and the pairs of all ranks (every rank calls it)."""
    import torch.distributed as dist
    t = torch.tensor([ms, pairs], dtype=torch.float64, device=device)
    if dist.is_initialized():
        m = t[:1].clone()
        dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
        p_ = t[1:].clone()
        dist.all_reduce(p_, op=dist.ReduceOp.SUM, group=group)
        return float(m.item()), float(p_.item())
    return ms, pairs


def bench_sharded(args):
    """N ranks (one per GPU) migrate ONE survey: rank r owns inline slab r of
    the output grid and migrates it from its halo traces (strong scaling; the
    step has no collective).  After the timed steps the slabs are gathered to
    every rank once and rank 0 checks the stitched image's fold against a
    one-plan migration of its own slab's columns."""
    import datetime
    import torch.distributed as dist
    from seisproc_b200 import _lib
    from seisproc_b200.sharding import ShardedPSTM
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    L = _lib.lib()
    s = make_workload(dev, 0, args)  # the same survey on every rank
    torch.cuda.synchronize()
    sh = ShardedPSTM(s.source_x, s.source_y, s.receiver_x, s.receiver_y, n_il=s.n_il,
                     n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x, origin_y=s.origin_y,
                     il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=s.xl_spacing, t0_ms=0.0,
                     dt_ms=s.dt_ms, n_samples=s.n_samples, in_t0_ms=0.0, in_dt_ms=s.dt_ms,
                     max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg,
                     velocity=torch.from_numpy(s.vrms), storage=args.storage, forward_only=True,
                     device=dev)
    local_tr = sh.local_traces(s.traces)
    img = fold = None
    for _ in range(args.warmup):
        sh.plan.load_traces(local_tr)
        img, fold = sh.plan.migrate_loaded(sh.velocity)
    sh.plan.check()
    pairs_local = float(fold[:, :sh.local_il].double().sum())
    dist.barrier()
    torch.cuda.synchronize()
    l0 = L.pstm_launch_count()
    with ClockSampler(local) as clk:
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            sh.plan.load_traces(local_tr)
            sh.plan.migrate_loaded(sh.velocity, image=img, fold=fold)
        e.record()
        torch.cuda.synchronize()
    launches = L.pstm_launch_count() - l0
    dist.barrier()
    ms, pairs_all = shard_aggregate(a.elapsed_time(e) / args.steps, pairs_local, dev)
    whole_fold = sh.gather(fold[:, :sh.local_il].contiguous())
    ok = bool(float(whole_fold.double().sum()) == pairs_all)
    if rank == 0:
        print(json.dumps({
            "metric": "PSTM Gpairs/s (out-sample x trace)",
            "value": pairs_all / (ms * 1e-3) / 1e9, "unit": "Gpairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": args.storage, "data": "synthetic",
            "config": {"workload": workload_name(args), "storage": args.storage,
                       "pairs_per_step": pairs_all,
                       "parallelism": f"inline slabs over {world} ranks: one survey, halo "
                                      "traces per slab, no collective in the step, slabs "
                                      "gathered once after timing",
                       "slab_inlines": [b - a_ for a_, b in sh.slabs],
                       "halo_traces_rank0": int(sh.halo.size),
                       "gathered_fold_matches_pairs": ok,
                       "l2": "inputs larger than L2; no flush"},
            "gpu_launches": int(launches * world), "clocks": clk.summary()}), flush=True)
    sh.close()
    dist.barrier()
    dist.destroy_process_group()


def bench_batched(args):
    """64 offset/azimuth classes (trace counts log-uniform 2k-40k), one persistent
    launch per step replayed from a CUDA graph; value = pairs of all classes / time.

    The line also carries the batched kernel's roofline (pairs / its CUDA-event
    time), ``error_vs_fp64`` of the run's storage and of the two others on
    checked classes, the reference port per class on a crop as the CPU baseline,
    and ``e2e``: every class from page-locked host buffers through
    ``MigrationEngine.migrate_bins_full`` into page-locked host images."""
    from seisproc_b200 import _lib
    from seisproc_b200.batched import BatchedPSTM
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    t_gen = time.perf_counter()
    surveys = batched_surveys(args, dev)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    s0 = surveys[0]
    n_t = s0.n_times
    vel = torch.from_numpy(s0.vrms).to(dev)
    t_tune = time.perf_counter()
    plans = class_plans(surveys, args.storage, args.variant, dev, vel)
    torch.cuda.synchronize()
    t_tune = time.perf_counter() - t_tune
    bufs = [s.traces for s in surveys]
    b = BatchedPSTM(plans, vel)
    b.capture(bufs)
    for _ in range(args.warmup):
        b.replay()
    torch.cuda.synchronize()
    b.check()
    pairs_c = [float(f.double().sum()) for f in b.folds]
    pairs = float(sum(pairs_c))
    l0 = L.pstm_launch_count()
    with ClockSampler(0) as clk:
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            b.replay()
        e.record()
        torch.cuda.synchronize()
    b.check()
    ms = a.elapsed_time(e) / args.steps
    launches = b.launches_per_replay * args.steps
    # the batched kernel alone (traces already staged): velocity check + persistent launch
    kms = []
    for _ in range(3):
        a.record()
        b.migrate()
        e.record()
        torch.cuda.synchronize()
        kms.append(a.elapsed_time(e))
    kernel_ms = statistics.median(kms)
    pk = peaks()
    peak_pairs = 148 * MUFU_PER_SM_CLK / RSQRT_PER_PAIR * pk["sm_max_mhz"] * 1e6 / 1e12
    achieved = pairs / (kernel_ms * 1e-3) / 1e12
    roof = {"bound": "mufu", "achieved": achieved, "peak": peak_pairs, "unit": "Tpairs/s",
            "frac": achieved / peak_pairs, "traffic": None, "mufu_per_pair": RSQRT_PER_PAIR,
            "traffic_note": "not captured for the batched launch",
            "peak_source": f"{pk['source']} sm_max_mhz {pk['sm_max_mhz']}",
            "kernel": "pstm_batch_kernel (persistent, all classes, fold counted in the launch)",
            "kernel_ms": kernel_ms}
    err, cb, e2e = None, None, None
    if not args.no_cpu:
        clusters = error_clusters(surveys[0].n_il, surveys[0].n_xl, args.err_clusters)
        chk = checked_classes(pairs_c)

        def check_images(images, folds, storage):
            return merge_checks([fp64_check(surveys[i], images[q].reshape(n_t, -1),
                                            folds[q].reshape(n_t, -1), clusters, False,
                                            args.aa_lmax, storage)
                                 for q, i in enumerate(chk)], storage)

        err = {args.storage: check_images([b.images[i] for i in chk], [b.folds[i] for i in chk],
                                          args.storage)}
        for st in ("f32", "bf16", "f16"):
            if st == args.storage:
                continue
            sub = class_plans([surveys[i] for i in chk], st, args.variant, dev, vel)
            bs = BatchedPSTM(sub, vel)
            bs.load([surveys[i].traces for i in chk])
            bs.migrate()
            torch.cuda.synchronize()
            bs.check()
            err[st] = check_images(bs.images, bs.folds, st)
            bs.close()
            for p_ in sub:
                p_.close()
        err["classes_checked"] = chk
        err["clusters_per_class"] = len(clusters)
        # CPU baseline: the reference port on a centred crop of every class
        cols = cpu_crop_columns(surveys[0], args.crop)
        ecol = torch.from_numpy(cols).to(dev)
        cp, csec, ncls = 0.0, 0.0, 0
        for i, sv in enumerate(surveys):
            pc = float(b.folds[i].reshape(n_t, -1)[:, ecol].double().sum())
            if pc <= 0:
                continue
            r = run_cpu_port(sv, cols, pc)
            cp += pc
            csec += r["seconds"]
            ncls += 1
        cb = {"value": cp / max(csec, 1e-12) / 1e9, "unit": "Gpairs/s",
              "cores": len(os.sched_getaffinity(0)), "kind": "port",
              "sample": f"every class with pairs in a centred {args.crop}x{args.crop}-column crop "
                        f"({ncls} classes, one bin at a time as the reference worker runs "
                        f"them), all of each class's traces supplied, {cp:.3e} pairs; constant "
                        "V = mean V_rms"}
    if not args.no_e2e:
        from seisproc_b200.engine import MigrationEngine
        host_bins = []
        for sv in surveys:
            t = torch.empty(tuple(sv.traces.shape), dtype=torch.float32, pin_memory=True)
            t.copy_(sv.traces)
            hb = {"traces": t.numpy()}
            for key in ("source_x", "source_y", "receiver_x", "receiver_y"):
                h = torch.empty(getattr(sv, key).shape, dtype=torch.float64, pin_memory=True)
                h.copy_(torch.from_numpy(getattr(sv, key)))
                hb[key] = h.numpy()
            host_bins.append(hb)
        host_v = torch.empty(s0.vrms.shape, dtype=torch.float32, pin_memory=True)
        host_v.copy_(torch.from_numpy(s0.vrms))
        shape = (n_t, s0.n_il, s0.n_xl)
        try:
            outs = [(torch.empty(shape, pin_memory=True), torch.empty(shape, pin_memory=True))
                    for _ in surveys]
            out_kind = "page-locked tensors"
        except RuntimeError:
            outs = [(np.empty(shape, np.float32), np.empty(shape, np.float32)) for _ in surveys]
            out_kind = "numpy arrays (page-locking the outputs failed)"
        eng = MigrationEngine(storage=args.storage, variant=args.variant)
        kw = dict(origin_x=s0.origin_x, origin_y=s0.origin_y, il_spacing=s0.il_spacing,
                  xl_spacing=s0.xl_spacing, azimuth_deg=0.0, n_il=s0.n_il, n_xl=s0.n_xl,
                  dt_ms=s0.dt_ms, t_min_ms=0.0, n_times=n_t, max_aperture_m=s0.max_aperture_m,
                  max_angle_deg=s0.max_angle_deg, normalize=True, velocity_model=host_v.numpy(),
                  out=outs)
        eng.migrate_bins_full(host_bins, **kw)
        calls = []
        for _ in range(max(2, min(args.steps, 3))):
            a.record()
            eng.migrate_bins_full(host_bins, **kw)
            e.record()
            torch.cuda.synchronize()
            calls.append(a.elapsed_time(e))
        e_ms = statistics.median(calls)
        h2d = sum(hb["traces"].nbytes + 4 * hb["source_x"].nbytes for hb in host_bins) \
            + host_v.numel() * 4
        e2e = {"value": pairs / (e_ms * 1e-3) / 1e9, "unit": "Gpairs/s",
               "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(2 * len(surveys) * int(np.prod(shape)) * 4),
               "ms_per_step": e_ms, "ms_calls": [round(c, 1) for c in calls],
               "api": "MigrationEngine.migrate_bins_full (plans, H2D, staging, batched launch, "
                      "fold normalisation, D2H of every class image and fold)",
               "outputs": out_kind}
        del outs
    n_tr = int(sum(sv.n_traces for sv in surveys))
    res = {"metric": "PSTM Gpairs/s (out-sample x trace), batched classes",
           "value": pairs / (ms * 1e-3) / 1e9, "unit": "Gpairs/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": args.storage, "data": "synthetic",
           "config": {"workload": f"batched 3D PSTM: {len(surveys)} offset/azimuth classes, "
                                  f"{n_tr} traces x {args.samples} samples, per-class "
                                  f"{args.grid}x{args.grid}x{args.samples} images, "
                                  f"{args.storage} storage, one persistent launch in a CUDA "
                                  "graph", "pairs_per_step": pairs, "datagen_s": t_gen,
                      "class_shapes": {str(k): b.shapes.count(k) for k in sorted(set(b.shapes))},
                      "class_shape_ids": b.shapes,
                      "shape_choice": ("autotuner per class (cached per problem class), "
                                       f"plans + choices {t_tune:.2f} s"
                                       if args.variant == "auto" else "fixed --variant"),
                      "launches_per_step": b.launches_per_replay,
                      "l2": "inputs larger than L2; no flush"},
           "roofline": roof, "error_vs_fp64": err, "cpu_baseline": cb, "e2e": e2e,
           "gpu_launches": int(launches), "clocks": clk.summary()}
    print(json.dumps(res), flush=True)
    b.close()
    for p_ in plans:
        p_.close()


def bench_batched_reference(args):
    """Reference arm of the batched config: the reference algorithm (CPU port)
    migrating the classes one bin at a time, as the reference worker does, on a
    centred crop of each class with all its traces supplied."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import pstm_fp64 as O
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    surveys = batched_surveys(args, dev)
    s0 = surveys[0]
    cols = cpu_crop_columns(s0, args.crop)
    il, xl = cols // s0.n_xl, cols % s0.n_xl
    cx = s0.origin_x + il * s0.il_spacing
    cy = s0.origin_y + xl * s0.xl_spacing
    t_ms = (np.arange(s0.n_times, dtype=np.float32) * np.float32(s0.dt_ms)).astype(np.float64)
    vmean = float(s0.vrms.mean())
    pcs = [O.count_pairs_fp64(sv.source_x, sv.source_y, sv.receiver_x, sv.receiver_y, cx, cy,
                              t_ms, vmean, sv.max_aperture_m, sv.max_angle_deg)
           for sv in surveys]
    vals, secs = [], []
    for it in range(args.warmup + args.steps):
        sec = sum(run_cpu_port(sv, cols, pc)["seconds"] for sv, pc in zip(surveys, pcs) if pc > 0)
        if it >= args.warmup:
            vals.append(sum(pcs) / sec / 1e9)
            secs.append(sec)
    v = statistics.median(vals)
    cb = {"value": v, "unit": "Gpairs/s", "cores": len(os.sched_getaffinity(0)), "kind": "port",
          "sample": f"every class with pairs in a centred {args.crop}x{args.crop}-column crop, "
                    f"one bin at a time, {sum(pcs):.3e} pairs; constant V = mean V_rms"}
    print(json.dumps({
        "metric": "PSTM Gpairs/s (out-sample x trace), batched classes", "value": v,
        "unit": "Gpairs/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.median(secs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"batched 3D PSTM: {len(surveys)} offset/azimuth classes, "
                               f"{args.samples} samples, per-class {args.grid}x{args.grid} "
                               "grids, the reference's one-bin-at-a-time loop on a crop"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "Gpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def bench_lsq(args):
    """Least-squares PSTM: 100x100x500 grid, 120k traces at 2 ms, FP32 -- dot-product
    test, finite-difference checks of the V gradient, 10 CG iterations."""
    from seisproc_b200 import synthetic
    from seisproc_b200.autograd import cgls, dot_product_test, migrate
    from seisproc_b200.kirchhoff import PSTMPlan
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    s = synthetic.survey_3d(n_traces=args.lsq_traces, seed=7, device=dev, n_samples=500, dt_ms=2.0,
                            extent=2500.0, max_offset=1500.0, n_il=100, n_xl=100, spacing=25.0,
                            n_diffractors=60, aperture=1000.0)
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                    in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg)
    v = torch.from_numpy(s.vrms).to(dev)
    a_, b_, rel = dot_product_test(plan, v, seed=7)
    # V-gradient directional derivatives vs central differences (relative step 1e-3)
    tr = s.traces
    g = torch.randn(v.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(3))
    vv = v.clone().requires_grad_(True)
    (migrate(tr, vv, plan) * g).sum().backward()
    rs = np.random.RandomState(20)
    fd, an = [], []
    tt = np.linspace(0.0, 1.0, s.n_times)[:, None, None]
    xx = np.linspace(0.0, 1.0, s.n_il)[None, :, None]
    yy = np.linspace(0.0, 1.0, s.n_xl)[None, None, :]
    for _ in range(args.fd_directions):
        # smooth random perturbation (keeps V t0 increasing in t0)
        c = rs.randn(4)
        f = (c[0] + c[1] * np.sin(np.pi * (tt + rs.rand())) + c[2] * np.cos(2 * np.pi * xx)
             + c[3] * np.sin(2 * np.pi * yy))
        dv = torch.from_numpy((f / np.abs(f).max()).astype(np.float32)).to(dev) * v * 1e-3
        f = lambda x: float((migrate(tr, x, plan).double() * g.double()).sum())
        fd.append((f(v + dv) - f(v - dv)) / 2.0)
        an.append(float((vv.grad.double() * dv.double()).sum()))
    fd, an = np.array(fd), np.array(an)
    plan.check()
    # the same geometry with band-limited noise-free data (8 Hz) and output
    # times from 200 ms: the forward map is smooth in V except at the linear
    # interpolation's sample kinks, so the finite differences should agree with
    # the gradient kernel to ~1e-2 (criterion); the noisy 30 Hz workload above
    # also crosses mask switches and kinks within the step
    sm = synthetic.survey_3d(n_traces=args.lsq_traces, seed=7, device=dev, n_samples=500,
                             dt_ms=2.0, extent=2500.0, max_offset=1500.0, n_il=100, n_xl=100,
                             spacing=25.0, n_diffractors=60, aperture=1000.0, f_peak=8.0,
                             noise_rel=0.0, n_times=400)
    cs = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
          for a in (sm.source_x, sm.source_y, sm.receiver_x, sm.receiver_y)]
    # an 89 deg angle limit: the aperture mask does not depend on V, so no mask
    # switches under the perturbation (the gradient holds the masks fixed)
    psm = PSTMPlan(*cs, n_il=sm.n_il, n_xl=sm.n_xl, n_times=400, origin_x=sm.origin_x,
                   origin_y=sm.origin_y, il_dx=sm.il_spacing, il_dy=0.0, xl_dx=0.0,
                   xl_dy=sm.xl_spacing, t0_ms=200.0, dt_ms=sm.dt_ms, n_samples=sm.n_samples,
                   in_t0_ms=0.0, in_dt_ms=sm.dt_ms, max_aperture_m=sm.max_aperture_m,
                   max_angle_deg=89.0)
    vs = torch.from_numpy(sm.vrms).to(dev)
    gs = torch.randn(vs.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(4))
    vsg = vs.clone().requires_grad_(True)
    (migrate(sm.traces, vsg, psm) * gs).sum().backward()
    rs2 = np.random.RandomState(21)
    fd2, an2 = [], []
    t2 = np.linspace(0.0, 1.0, 400)[:, None, None]
    for _ in range(args.fd_directions):
        # smooth random direction (V t0 stays increasing in t0)
        c = rs2.randn(4)
        f = (c[0] + c[1] * np.sin(np.pi * (t2 + rs2.rand())) + c[2] * np.cos(2 * np.pi * xx)
             + c[3] * np.sin(2 * np.pi * yy))
        dv = torch.from_numpy((f / np.abs(f).max()).astype(np.float32)).to(dev) * vs * 1e-3
        f2_ = lambda x: float((migrate(sm.traces, x, psm).double() * gs.double()).sum())
        fd2.append((f2_(vs + dv) - f2_(vs - dv)) / 2.0)
        an2.append(float((vsg.grad.double() * dv.double()).sum()))
    fd2, an2 = np.array(fd2), np.array(an2)
    psm.check()
    psm.close()
    del sm, cs
    d = plan.demigrate(migrate(tr, v, plan), v)  # data in the range of L
    m, hist = cgls(plan, d, v, n_iter=args.cg_iters)
    it_s = [h[2] for h in hist[1:]]
    print(json.dumps({
        "metric": "LSQ PSTM CG seconds per iteration", "value": float(np.median(it_s)),
        "unit": "s/iter", "n_gpus": 1, "higher_is_better": False, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"least-squares PSTM 100x100x500, {args.lsq_traces // 1000}k "
                               "traces at 2 ms, FP32", "cg_iterations": args.cg_iters},
        "dot_product": {"<Lm,d>": a_, "<m,L^T d>": b_, "rel": rel},
        "vgrad_fd": {"directions": args.fd_directions,
                     "rel_l2": float(np.linalg.norm(fd - an) / np.linalg.norm(fd))
                     if args.fd_directions else None,
                     "note": "noisy 30 Hz data from t0 = 0: includes interpolation kinks and "
                             "mask switches"},
        "vgrad_fd_smooth": {"directions": args.fd_directions,
                            "rel_l2": float(np.linalg.norm(fd2 - an2) / np.linalg.norm(fd2))
                            if args.fd_directions else None, "criterion": 1e-2,
                            "note": "same geometry and size, 8 Hz noise-free data, output "
                                    "times 200-998 ms, 1000 m aperture with an 89 deg angle "
                                    "limit (no V-dependent mask), smooth random "
                                    "perturbations of relative size 1e-3"},
        "cg": {"residual_history": [h[1] for h in hist], "misfit_reduction": hist[-1][1]},
    }), flush=True)
    plan.close()


def velocity_case(n_t: int, n: int):
    """The velocity config's picked cube (43 x 23 x 23 nodes: every 100 ms and
    250 m, seeded) and the output grid's times and column coordinates."""
    rs = np.random.RandomState(5)
    z = np.linspace(0.0, 4.2, 43).astype(np.float32)          # picks every 100 ms
    x = np.linspace(-250.0, 5250.0, 23).astype(np.float32)    # nodes every 250 m
    y = np.linspace(-250.0, 5250.0, 23).astype(np.float32)
    cube = (1500 + 500 * z[:, None, None] + 0.02 * x[None, :, None] + 0.01 * y[None, None, :]
            + rs.uniform(-25, 25, (z.size, x.size, y.size))).astype(np.float32)
    t_s = np.arange(n_t) * 0.004
    il = np.arange(n)[:, None]
    xl = np.arange(n)[None, :]
    cx = (12.5 + 25.0 * il + 0 * xl).ravel()
    cy = (12.5 + 0 * il + 25.0 * xl).ravel()
    return z, x, y, cube, t_s, cx, cy


def bench_velocity_reference(args):
    """Reference arm of the velocity config: the reference's evaluation
    (models/velocity_model.py:181-245, scipy RegularGridInterpolator, linear,
    extrapolating) at every output time of every 50th column, on rank 0."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from scipy.interpolate import RegularGridInterpolator
    n_t, n = args.samples, args.grid
    z, x, y, cube, t_s, cx, cy = velocity_case(n_t, n)
    sel = np.arange(0, n * n, 50)
    f = RegularGridInterpolator((z, x, y), cube, method="linear", bounds_error=False,
                                fill_value=None)
    pts = np.stack(np.broadcast_arrays(t_s[:, None], cx[sel][None, :], cy[sel][None, :]),
                   -1).reshape(-1, 3)
    vals, secs = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        f(pts).astype(np.float32)
        sec = time.perf_counter() - t0
        if i >= args.warmup:
            vals.append(pts.shape[0] / sec / 1e9)
            secs.append(sec)
    v = statistics.median(vals)
    print(json.dumps({
        "metric": "V_rms grid Gsamples/s", "value": v, "unit": "Gsamples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.median(secs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 blend, f32 out",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"3-D velocity cube {z.size}x{x.size}x{y.size} nodes resampled "
                               f"onto the {n}x{n}x{n_t} output grid"},
        "cpu_baseline": {"value": v, "unit": "Gsamples/s", "cores": 1, "kind": "port",
                         "sample": f"{sel.size} of {n * n} columns x {n_t} times, scipy "
                                   "RegularGridInterpolator"},
        "e2e": {"value": v, "unit": "Gsamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def bench_unavailable(why: str):
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)


def bench_velocity(args):
    """V_rms ingestion: a picked 3-D velocity cube (coarse nodes, as an
    IL-XL-T-V or SEG-Y velocity file gives) resampled onto every sample of the
    3D output grid (1000 x 200 x 200) by pstm_velocity_grid.  value = output
    samples per second of the kernel with the model and tables resident;
    roofline = its 4 written bytes per sample against HBM; e2e = the whole
    velocity_grid() call (host tables, uploads, kernel); cpu_baseline = the
    float64 numpy restatement on a column sample."""
    from seisproc_b200 import _lib
    from seisproc_b200 import models as M
    from seisproc_b200.velocity_io import VelocityGridder, velocity_grid
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    n_t, n = args.samples, args.grid
    z, x, y, cube, t_s, cx, cy = velocity_case(n_t, n)
    m = M.create_3d_velocity(cube, z, x, y)
    g = VelocityGridder(m, t_s, cx, cy, dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MB > L2
    for _ in range(args.warmup):
        g.run()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    l0 = L.pstm_launch_count()
    with ClockSampler(0) as clk:
        for a, b in ev:
            flush.zero_()
            a.record()
            g.run()
            b.record()
        torch.cuda.synchronize()
    launches = L.pstm_launch_count() - l0
    ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    samples = float(n_t * n * n)
    # e2e: the public call, host tables + uploads + kernel + D2H of the grid
    e2e_ms = []
    for _ in range(max(3, min(args.steps, 5))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = velocity_grid(m, t_s, cx, cy, dev).cpu()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.median(e2e_ms)
    ok = np.array_equal(out.numpy(), g.out.cpu().numpy())
    # CPU: the float64 numpy restatement on every 50th column
    sel = np.arange(0, n * n, 50)
    t0 = time.perf_counter()
    host = m.rms_grid(t_s, cx[sel], cy[sel])
    cpu_s = time.perf_counter() - t0
    dv = g.out.cpu().numpy()[:, sel]
    ulps = int(np.abs(dv.view(np.int32).astype(np.int64) -
                      host.view(np.int32).astype(np.int64)).max())
    pk = peaks()
    gbs = samples * 4 / (ms * 1e-3) / 1e9
    print(json.dumps({
        "metric": "V_rms grid Gsamples/s", "value": samples / (ms * 1e-3) / 1e9,
        "unit": "Gsamples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 blend, f32 out", "data": "synthetic",
        "config": {"workload": f"3-D velocity cube {z.size}x{x.size}x{y.size} nodes resampled "
                               f"onto the {n}x{n}x{n_t} output grid",
                   "l2": "256 MB buffer written between timed launches"},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": gbs / pk["hbm_gbs"], "traffic": None,
                     "algorithmic_bytes_per_sample": 4, "peak_source": pk["source"]},
        "e2e": {"value": samples / (e2e * 1e-3) / 1e9, "unit": "Gsamples/s",
                "h2d_bytes_per_step": int(cube.nbytes + 12 * n_t + 24 * n * n),
                "d2h_bytes_per_step": int(samples * 4), "ms_per_step": e2e,
                "matches_resident_run": ok},
        "cpu_baseline": {"value": sel.size * n_t / cpu_s / 1e9, "unit": "Gsamples/s", "cores": 1,
                         "kind": "port", "sample": f"{sel.size} of {n * n} columns x {n_t} "
                                                   "times, float64 numpy"},
        "max_ulps_vs_host": ulps, "gpu_launches": int(launches), "clocks": clk.summary(),
    }), flush=True)


TR_SPACING, TR_DT, TR_APERTURE, TR_ANGLE = 25.0, 4.0, 1000.0, 60.0
TR_V0, TR_GRADIENT = 1500.0, 0.6


def time_rms_survey(n_tr: int, n_s: int):
    """The time_rms workload's seeded traces and coordinates (float32 numpy):
    midpoints uniform over 5 x 5 km, offsets uniform 0-3 km, azimuths uniform,
    Gaussian traces (n_s, n_tr)."""
    rs = np.random.RandomState(2025)
    mx, my = rs.uniform(0, 5000, n_tr), rs.uniform(0, 5000, n_tr)
    off, phi = rs.uniform(0, 3000, n_tr), rs.uniform(0, 2 * np.pi, n_tr)
    sx = (mx - 0.5 * off * np.cos(phi)).astype(np.float32)
    sy = (my - 0.5 * off * np.sin(phi)).astype(np.float32)
    rx = (mx + 0.5 * off * np.cos(phi)).astype(np.float32)
    ry = (my + 0.5 * off * np.sin(phi)).astype(np.float32)
    tr = rs.standard_normal((n_s, n_tr)).astype(np.float32)
    return tr, sx, sy, rx, ry


def time_rms_workload(n_tr: int, n_s: int, n: int) -> str:
    return (f"time-domain RMS operator, {n_tr} traces x {n_s} samples, {n}x{n}x{n_s} output "
            f"grid, aperture {TR_APERTURE:.0f} m, {TR_ANGLE:.0f} deg, tiles of 100 points, "
            "5000-trace cap")


def time_rms_cpu_sample(tr, sx, sy, rx, ry, n: int, n_s: int):
    """The reference's time-domain computation on the host cores (the oracle's
    bit-identical torch port, all threads) on a bounded sample of the time_rms
    workload: its first tile (100 output points) with every trace the
    reference lists for it.  Returns (evaluated triples, seconds, description,
    threads); triples count the (point, trace) pairs inside the aperture times
    the input samples, as the kernel's metric does."""
    import torch as _t
    from oracle import time_domain as otd
    from seisproc_b200.velocity import VelocityModel
    threads = len(os.sched_getaffinity(0))
    _t.set_num_threads(threads)
    f32 = np.float32
    ox, oy = otd.output_grid_f32(12.5, 12.5, TR_SPACING, TR_SPACING, 0.0, n, n)
    tile = otd.effective_tile_size(100, 5000, 200)
    mx, my = (sx + rx) / f32(2), (sy + ry) / f32(2)
    (_, _, sel), = otd.tile_trace_lists(ox[:tile], oy[:tile], mx, my, tile, TR_APERTURE, 5000)
    if sel.size == 0:
        raise RuntimeError("the first tile lists no traces")
    pts = np.arange(min(tile, n * n))
    hh = np.sqrt((ox[pts, None] - mx[None, sel]) ** 2 + (oy[pts, None] - my[None, sel]) ** 2)
    evals = int((hh < TR_APERTURE).sum()) * n_s
    t_in = _t.arange(n_s, dtype=_t.float32) * TR_DT
    v_in = VelocityModel("gradient", TR_V0, gradient=TR_GRADIENT).rms_velocity_at_time(t_in)
    t0 = time.perf_counter()
    otd.time_domain_rms_torch_port(tr, sx, sy, rx, ry, ox, oy, n_s, v_in.numpy(), TR_DT, 0.0,
                                   TR_APERTURE, TR_ANGLE, n, n, 12.5, 12.5, TR_SPACING,
                                   TR_SPACING, 0.0, first_tile=0, n_tiles=1)
    sec = time.perf_counter() - t0
    return evals, sec, (f"first tile: {pts.size} points x its {sel.size} listed traces x "
                        f"{n_s} samples, the reference's float32 torch loop (oracle port), "
                        f"{threads} threads"), threads


def bench_time_rms_reference(args):
    """Reference arm of the time_rms config: the reference's float32 torch
    loop (the oracle's bit-identical port, kind "port"; the reference itself
    does not travel) on the bounded sample of ``time_rms_cpu_sample``, one
    sample per step, all host threads, on rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    n_tr, n_s, n = args.traces, args.samples, args.grid
    tr, sx, sy, rx, ry = time_rms_survey(n_tr, n_s)
    vals, secs = [], []
    for i in range(args.warmup + args.steps):
        ev, sec, sample, threads = time_rms_cpu_sample(tr, sx, sy, rx, ry, n, n_s)
        if i >= args.warmup:
            vals.append(ev / sec / 1e9)
            secs.append(sec)
    v = statistics.median(vals)
    print(json.dumps({
        "metric": "time-domain RMS scatter Gevals/s", "value": v, "unit": "Gevals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.median(secs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference", "config": {"workload": time_rms_workload(n_tr, n_s, n)},
        "cpu_baseline": {"value": v, "unit": "Gevals/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "Gevals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def bench_time_rms(args):
    """The time-domain RMS operator (MigrationEngine.migrate_bin_time_domain_rms)
    on the 3D survey's geometry: N traces with midpoints over 5 x 5 km, offsets
    up to 3 km, V_rms with a linear gradient, the 200 x 200 x 1000 output grid
    at 25 m, aperture 1000 m, 60 deg, time-dependent aperture, the reference's
    default tiles (100 points) and trace cap (5000 per tile).
    value = evaluated (output point, trace, input sample) triples per second of
    pstm_time_rms_migrate with inputs resident (points within the aperture
    only: the kernel skips the others before the sample loop); roofline = 8
    MUFU operations per triple (five IEEE divisions, three IEEE square roots);
    e2e = the whole engine call from host arrays; cpu_baseline = the float32
    oracle on one tile."""
    from seisproc_b200 import _lib
    from seisproc_b200 import time_domain as TD
    from seisproc_b200.engine import MigrationEngine
    from seisproc_b200.velocity import VelocityModel
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    n_tr, n_s, n = args.traces, args.samples, args.grid
    sp, dt, A, theta = TR_SPACING, TR_DT, TR_APERTURE, TR_ANGLE
    tr, sx, sy, rx, ry = time_rms_survey(n_tr, n_s)
    vm = VelocityModel("gradient", TR_V0, gradient=TR_GRADIENT)
    grid = dict(origin_x=12.5, origin_y=12.5, il_spacing=sp, xl_spacing=sp, azimuth_deg=0.0,
                n_il=n, n_xl=n, dt_ms=dt, t_min_ms=0.0, n_times=n_s)
    # resident inputs, built once as the engine builds them
    f32 = torch.float32
    d_tr = torch.from_numpy(tr).to(dev)
    g = [torch.from_numpy(a).to(dev) for a in (sx, sy, rx, ry)]
    il = torch.arange(n, device=dev, dtype=f32) * sp
    xl_g, il_g = torch.meshgrid(il, il, indexing="xy")
    ox = (12.5 + il_g.flatten()).contiguous()
    oy = (12.5 + xl_g.flatten()).contiguous()
    t_axis = torch.arange(n_s, device=dev, dtype=f32) * dt
    tile = TD.effective_tile_size(100, 5000, 200)
    mid_x, mid_y, hoff_sq, col = TD.trace_geometry(*g, 12.5, 12.5, sp, sp, 0.0, n, n)
    p_tile, p_trace = TD.tile_pairs(ox, oy, mid_x, mid_y, tile, A, 5000)
    pairs = TD.column_pairs(ox, oy, mid_x, mid_y, col, tile, A, 5000)
    v_in = vm.rms_velocity_at_time(t_axis)
    k_img = torch.empty((n_s, n * n), dtype=f32, device=dev)
    k_fold = torch.empty_like(k_img)
    # algorithmic work: (pair, point) with h < A, times the input samples
    evals = 0
    for a in range(0, p_tile.numel(), 1 << 18):
        pt, pj = p_tile[a:a + (1 << 18)], p_trace[a:a + (1 << 18)]
        pts = pt[:, None] * tile + torch.arange(tile, device=dev)[None, :]
        ok = pts < n * n
        pts = pts.clamp(max=n * n - 1)
        h = torch.sqrt((ox[pts] - mid_x[pj][:, None]) ** 2 + (oy[pts] - mid_y[pj][:, None]) ** 2)
        evals += int(((h < A) & ok).sum())
    evals *= n_s

    def run():
        return TD.migrate_kirchhoff_time_domain_rms(
            d_tr, *g, ox, oy, t_axis, vm, dt, 0.0, A, theta, n, n, 12.5, 12.5, sp, sp, 0.0)

    def kernel():
        TD.launch_time_rms(d_tr, mid_x, mid_y, hoff_sq, ox, oy, v_in, pairs, tile, dt, 0.0, A,
                           theta, True, k_img, k_fold)

    for _ in range(args.warmup):
        kernel()
    torch.cuda.synchronize()
    # value: the kernel with its pair list and inputs resident (one launch per step)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    l0 = L.pstm_launch_count()
    with ClockSampler(0) as clk:
        for a, b in ev:
            a.record()
            kernel()
            b.record()
        torch.cuda.synchronize()
    launches = L.pstm_launch_count() - l0
    kern_ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    # the whole tensor-level call (pair selection + V_rms table + kernel)
    run()
    torch.cuda.synchronize()
    cev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(max(2, min(args.steps, 3)))]
    for a, b in cev:
        a.record()
        img_call, fold_call = run()
        b.record()
    torch.cuda.synchronize()
    call_ms = statistics.median(a.elapsed_time(b) for a, b in cev)
    same = bool(torch.equal(fold_call.reshape(n_s, -1), k_fold))
    # e2e: the engine call from host arrays (H2D, plan, kernel, D2H)
    eng = MigrationEngine()
    e2e_ms = []
    for _ in range(max(2, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img, fold = eng.migrate_bin_time_domain_rms(
            tr, sx, sy, rx, ry, velocity_model=vm, max_aperture_m=A, max_angle_deg=theta,
            normalize=False, **grid)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.median(e2e_ms)
    # CPU: the float32 oracle on a sample of the same workload
    cpu = None
    if not args.no_cpu:
        ev_cpu, cpu_s, sample, threads = time_rms_cpu_sample(tr, sx, sy, rx, ry, n, n_s)
        cpu = {"value": ev_cpu / cpu_s / 1e9, "unit": "Gevals/s", "cores": threads,
               "kind": "port", "sample": sample}
    pk = peaks()
    mufu_peak = 148 * 16 * pk["sm_max_mhz"] * 1e6 / 8 / 1e9  # Gevals/s
    val = evals / (kern_ms * 1e-3) / 1e9
    print(json.dumps({
        "metric": "time-domain RMS scatter Gevals/s", "value": val, "unit": "Gevals/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": kern_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": time_rms_workload(n_tr, n_s, n),
                   "pairs": int(p_tile.numel()), "evals": evals,
                   "l2": "inputs (traces 2 GB) larger than L2"},
        "call_ms": call_ms, "call_fold_matches_kernel_run": same,
        "roofline": {"bound": "mufu", "achieved": val, "peak": mufu_peak, "unit": "Gevals/s",
                     "frac": val / mufu_peak, "traffic": None,
                     "mufu_per_eval": 8, "peak_source": pk["source"]},
        "e2e": {"value": evals / (e2e * 1e-3) / 1e9, "unit": "Gevals/s",
                "h2d_bytes_per_step": int(tr.nbytes + 16 * n_tr),
                "d2h_bytes_per_step": int(2 * 4 * n * n * n_s), "ms_per_step": e2e},
        "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk.summary(),
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16"])
    ap.add_argument("--variant", default="auto",
                    help="kernel shape id, 0 for the library's heuristic, or auto (the tuner's "
                         "choice per problem class)")
    ap.add_argument("--traces", type=int, default=500_000)
    ap.add_argument("--samples", type=int, default=1000)
    ap.add_argument("--grid", type=int, default=200)
    ap.add_argument("--crop", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--err-crop", type=int, default=2,
                    help="anti-alias workload: side of the centred crop the FP64 oracle is "
                         "timed on as the CPU baseline")
    ap.add_argument("--err-clusters", type=int, default=16,
                    help="2x2 column clusters checked against the FP64 oracle (>= 9: corners, "
                         "edge midpoints and centre come first)")
    ap.add_argument("--antialias", action="store_true",
                    help="triangle anti-alias filter (half-width from the operator dip)")
    ap.add_argument("--aa-lmax", type=float, default=32.0)
    ap.add_argument("--utm", action="store_true",
                    help="world coordinates offset by a UTM origin (5e5, 6e6) m")
    ap.add_argument("--shard-mode", default="auto", choices=["auto", "slabs", "replicas"],
                    help="auto: inline slabs of one survey when N > 1 ranks (strong scaling), "
                         "the single-plan path on one; slabs: the slab path at any N (one "
                         "slab = the whole grid on one rank); replicas: one independent "
                         "survey per rank (weak scaling)")
    ap.add_argument("--classes", type=int, default=64,
                    help="batched config: the first N of the 64 offset/azimuth classes")
    ap.add_argument("--lsq-traces", type=int, default=120_000)
    ap.add_argument("--cg-iters", type=int, default=10)
    ap.add_argument("--fd-directions", type=int, default=20)
    ap.add_argument("--config", default="3d",
                    choices=["3d", "batched", "lsq", "velocity", "time_rms"])
    args = ap.parse_args()
    if args.variant != "auto":
        args.variant = int(args.variant)
    if args.config == "batched":
        return bench_batched(args) if args.impl == "ours" else bench_batched_reference(args)
    if args.config == "lsq":
        if args.impl == "ours":
            return bench_lsq(args)
        return bench_unavailable("the reference has no demigration (adjoint) and no "
                                 "least-squares migration")
    if args.config == "velocity":
        return bench_velocity(args) if args.impl == "ours" else bench_velocity_reference(args)
    if args.config == "time_rms":
        return bench_time_rms(args) if args.impl == "ours" else bench_time_rms_reference(args)
    if args.impl == "reference":
        bench_reference(args)
    elif args.shard_mode == "slabs" or (args.shard_mode == "auto" and
                                         int(os.environ.get("WORLD_SIZE", "1")) > 1):
        bench_sharded(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
