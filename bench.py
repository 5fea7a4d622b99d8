"""Benchmark of the ARGOT point-source RT hot path on B200.

One step = one pass of the hot path over one synthetic workload with its
inputs resident in HBM: the march of every light ray (calc_optical_depth,
FP32 with Kahan columns), the stitching of columns into rays, and the
per-cell photo-ionisation / heating rates (calc_photoion_rate; FP32 exact
quadrature by default).  Rays are generated on the device by the tree walk
before timing (the producer step of the path).

Default workload: 256^3 lognormal mesh (sigma_ln 1.2), 4096 clustered
sources, theta 0.5 -- the largest single-GPU configuration, on which the
target throughput is quoted.  Inputs (13 GB of rays + a 268 MB field) are
larger than the 126 MB L2, so no flush is needed between steps.

metric: ray-cell crossings/s of the whole step; the JSON line also carries
Gamma-cells/s, the per-kernel split, a roofline object for the march (HBM
bound) and the reference's CPU path timed on a bounded sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W]
                       [--impl ours|reference] [--config largest|plain|...]
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CONFIGS = ("largest", "plain", "precision", "learned", "tiny", "plain256", "batched", "batched_small",
           "ionized", "ionized64", "art", "art256", "art64")
ART_METRIC = "ART diffuse ray-cell steps/s (768 HEALPix directions, 1 B200)"
ART_UENETOK = 1.0e4
METRIC = "ray-cell crossings/s (march+stitch+rates, 1 B200)"
# DRAM bytes per ray-cell crossing of k_march_rays<Kahan> measured by ncu on
# the 256^3 / 16-source case (dram__bytes_read.sum + dram__bytes_write.sum =
# 104.7 + 17.4 GB over a 104.1 ms launch for 6.030e10 crossings); the
# workloads here are too large to capture, so `traffic` scales this figure.
MARCH_DRAM_BYTES_PER_CROSSING = 2.024
# the same capture's L2 bytes (lts__t_sectors.sum x 32 B, 413.0 GB over the
# launch's 6.030e10 crossings): what the L2 serves per crossing
MARCH_L2_BYTES_PER_CROSSING = 6.848
UNIT = "crossings/s"


def make_workload(name: str, rank: int = 0):
    from argot_b200 import workload as W
    seed_shift = 1000 * rank
    if name == "largest":
        return W.largest(seed=5 + seed_shift)
    if name == "plain":
        return W.plain(seed=1 + seed_shift)
    if name == "precision":
        return W.precision(seed=2 + seed_shift)
    if name == "learned":
        return W.learned(seed=4 + seed_shift)
    if name == "tiny":
        return W.tiny(32, 16, seed=7 + seed_shift)
    if name == "plain256":
        # profiling case: a field larger than L2 with few rays (~4 GB on the device)
        return W.plain(edge=256, nsrc=16, seed=1 + seed_shift)
    if name == "ionized":
        # fully ionised 128^3 (thin rays): where the surrogate can serve rays
        return W.ionized(128, 256, seed=9 + seed_shift)
    if name == "ionized64":
        # profiling case for the surrogate kernels (fills the GPU, ~1 GB on the device)
        return W.ionized(64, 64, seed=9 + seed_shift)
    if name == "art":
        # the diffuse-radiation path on the precision mesh (128^3)
        return W.precision(seed=2 + seed_shift)
    if name == "art256":
        return W.largest(seed=5 + seed_shift)
    if name == "art64":
        # profiling case for the ART kernels
        return W.plain(seed=1 + seed_shift)
    if name == "batched":
        return W.batched(48, seed=3 + seed_shift)
    if name == "batched_small":
        return W.batched(12, seed=3 + seed_shift, edges=(16, 24, 32))
    raise ValueError(name)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def workload_config(wl, ws: int, sharded: bool) -> dict:
    """The `config` of a bench line: what defines the workload, the same in
    both arms (the run's own details go to `run`)."""
    return {"workload": wl.name, "mesh": f"{wl.edge}^3", "sources": wl.nsrc, "theta": wl.theta,
            "l2": "inputs larger than L2 (rays and fields of the whole problem); no flush",
            "parallelism": (f"{ws} ranks, target x-slabs of one problem, rate slabs all-gathered"
                            if sharded else f"{ws} independent problems (one per rank)")}


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle
    reasons); reading settings only."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws, x: float, device=None) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(ws, x: float, device=None) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------ CPU baseline
def reference_setup(wl, threads: int | None = None):
    """ARGOT's own C (the reference build for this mesh edge) loaded with the
    workload's mesh and sources; the reference builds its own tree."""
    from oracle.oracle import RefLib
    threads = threads or os.cpu_count() or 1
    R = RefLib(wl.edge)
    R.init(wl.lunit, wl.denstonh, wl.theta, threads)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    R.threads = threads
    return R


def cpu_sample(wl, target_seconds: float = 15.0, max_cells: int = 1 << 20, R=None, seed: int = 0):
    """The reference's hot path on a bounded, seeded sample of target cells:
    one contiguous group of target cells, the reference's own grouping unit,
    sized by a short probe to take about `target_seconds`.  Returns
    crossings/s over calc_optical_depth + accum_optical_depth +
    calc_photoion_rate."""
    from oracle.oracle import Oracle, unit_box_grid
    if R is None:
        R = reference_setup(wl)
    threads = R.threads
    rng = np.random.default_rng(seed)
    ncell = wl.edge ** 3
    # size the group by a short probe, then run it
    ncells = min(256, ncell)
    im0 = int(rng.integers(0, ncell - ncells + 1))
    R.zero_rates()
    t0 = time.time()
    probe = R.run_range(im0, im0 + ncells, True, want=("seg",))
    dt = max(time.time() - t0, 1e-3)
    ncells = int(min(max_cells, ncell, max(64, ncells * target_seconds / dt)))
    im0 = int(rng.integers(0, ncell - ncells + 1))
    R.zero_rates()
    out = R.run_range(im0, im0 + ncells, True, want=("seg",))
    times = out["times"]
    o = Oracle()
    cross = float(o.count_crossings(unit_box_grid(wl.edge, wl.lunit, wl.denstonh), out["seg"]).sum())
    hot = float(times[1] + times[2] + times[3])
    return {"value": cross / hot, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": (f"{ncells} consecutive target cells from index {im0} of {wl.name} "
                       f"({out['nray']} rays, {cross:.3e} crossings); hot-path wall "
                       f"{hot:.2f} s (march {times[1]:.2f}, accum {times[2]:.3f}, "
                       f"rates {times[3]:.2f})"),
            "march_crossings_per_s": cross / times[1] if times[1] > 0 else None,
            "gamma_cells_per_s": ncells / times[3] if times[3] > 0 else None,
            "wall_s": hot,
            "_probe_rays": probe["nray"]}


def reference_gpu_sample(wl, target_rays: int = 2_000_000, seed: int = 1, reps: int = 3):
    """ARGOT's own GPU entry points (calc_optical_depth_cuda,
    calc_photoion_rate_cuda; compiled for sm_100a with the reference's nvcc
    flags) on a bounded, seeded sample of the same workload: one contiguous
    range of target cells holding about `target_rays` rays (the reference
    keeps a 2 KB spectrum per ray in host and device memory, which bounds the
    sample), run group by group as calc_ARGOT_part runs it.  Reported: the
    hot path through the reference's calls (wall: its allocations, host
    copies, transfers and kernels; accum_optical_depth on the host) and its
    two kernels alone (CUDA events, the reference's launch geometry)."""
    from oracle.oracle import Oracle, RefGpu, unit_box_grid
    R = RefGpu(wl.edge)
    try:
        R.init(wl.lunit, wl.denstonh, wl.theta, os.cpu_count() or 1)
        R.set_mesh(*wl.fields())
        R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
        R.upload()
        rng = np.random.default_rng(seed)
        ncell = wl.edge ** 3
        probe = min(256, ncell)
        im0 = int(rng.integers(0, ncell - probe + 1))
        per_cell = max(1.0, R.count_rays(im0, im0 + probe) / probe)
        ncells = int(min(ncell, max(64, target_rays / per_cell)))
        im0 = int(rng.integers(0, ncell - ncells + 1))
        R.zero_rates_gpu()
        R.run_range_gpu(im0, im0 + ncells, kernel_reps=0)  # warm-up (module loading)
        R.zero_rates_gpu()
        out = R.run_range_gpu(im0, im0 + ncells, kernel_reps=reps, want=("seg",))
        ref_rates = R.rates_gpu()
        # the same loop with this library's drop-in entry points linked in
        from argot_b200 import _lib as L
        R.use_entry_points(L.load())
        # a first pass warms the library's pools and modules; the second is
        # timed (the reference's entry points allocate on every call anyway)
        R.zero_rates_gpu()
        R.run_range_gpu(im0, im0 + ncells, kernel_reps=0)
        R.zero_rates_gpu()
        ours = R.run_range_gpu(im0, im0 + ncells, kernel_reps=0)
        our_rates = R.rates_gpu()
        R.use_entry_points(None)
    finally:
        R.close()
    cross = float(Oracle().count_crossings(unit_box_grid(wl.edge, wl.lunit, wl.denstonh), out["seg"]).sum())
    calls = out["march_s"] + out["accum_s"] + out["rates_s"]
    ours_calls = ours["march_s"] + ours["accum_s"] + ours["rates_s"]
    nz = ref_rates != 0
    drop = {"what": "the same loop (reference tree, host light rays) with libargot_b200's "
                    "calc_optical_depth_cuda / calc_photoion_rate_cuda linked in",
            "value": cross / ours_calls, "unit": UNIT,
            "calls_s": {"calc_optical_depth_cuda": ours["march_s"], "accum_optical_depth": ours["accum_s"],
                        "calc_photoion_rate_cuda": ours["rates_s"]},
            "max_rel_diff_vs_reference_gpu": (float(np.max(np.abs(our_rates[nz].astype(np.float64) -
                                                                  ref_rates[nz]) / np.abs(ref_rates[nz])))
                                              if nz.any() else None)}
    t_mk, t_rk = out["march_kernel_ms"] / 1e3, out["rate_kernel_ms"] / 1e3
    hbm, _, peak_kind = measured_peaks()
    march_gbs = (16.0 * cross + 36.0 * out["nseg"]) / t_mk / 1e9
    return {"kind": "reference",
            "build": "ARGOT src/calc_optical_depth_cuda.cu, src/calc_photoion_rate_cuda.cu, "
                     "nvcc -use_fast_math -O3 for sm_100a",
            "sample": (f"{ncells} consecutive target cells from index {im0} of {wl.name} "
                       f"({out['nray']} rays, {cross:.3e} crossings, {out['groups']} groups)"),
            "value": cross / calls, "unit": UNIT,
            "kernels_value": cross / (t_mk + t_rk),
            "march_crossings_per_s": cross / t_mk,
            "march_roofline": {"achieved": march_gbs, "peak": hbm, "unit": "GB/s", "frac": march_gbs / hbm,
                               "peak_kind": f"{peak_kind} hbm_gbs", "bytes_model": "16 B per crossing + 36 B per ray"},
            "gamma_cells_per_s": ncells / t_rk,
            "rates_rays_per_s": out["nray"] / t_rk,
            "calls_s": {"calc_optical_depth_cuda": out["march_s"], "accum_optical_depth": out["accum_s"],
                        "calc_photoion_rate_cuda": out["rates_s"], "ray_setup_host": out["setup_s"]},
            "kernels_s": {"calc_optical_depth_kernel": t_mk, "calc_photoion_rate_kernel": t_rk},
            "dropin": drop}


# ------------------------------------------------------------ rate modes
def load_surrogate(pb):
    """The trained weights (argot_b200/data/surrogate.npz) on the device and
    the emitters' blackbody integrals; None when no weights are present."""
    from argot_b200 import surrogate as S
    if not os.path.exists(S.WEIGHTS):
        return None
    pb.set_blackbody()
    return S.Surrogate.from_file()


def compare_rate_modes(pb, rays, tau, prec, sur):
    """One pass of each rate kernel over every group after the same march:
    device time of each (CUDA events around the rate launches only).  Their
    errors come from `sampled_parity` (against the FP64 CPU oracle)."""
    import torch
    from argot_b200 import _lib as L
    dev = pb.device
    modes = [("exact_f64", L.RATE_EXACT_F64), ("exact_f32", L.RATE_EXACT_F32)]
    if sur is not None:
        modes.append(("surrogate", None))
    fields = {m: torch.zeros(6 * pb.ncell, dtype=torch.float32, device=dev) for m, _ in modes}
    t = {m: 0.0 for m, _ in modes}
    counters = torch.zeros(2, dtype=torch.int64, device=dev)
    single = len(pb.groups) == 1
    if sur is not None and getattr(pb, "_sur_work", None) is None:
        pb._sur_work = pb.surrogate_work()  # allocated outside the timed passes
    from argot_b200.pipeline import RayGroup
    for gi, g in enumerate(pb.groups):
        if not single:
            pb.emit(g, rays)
        pb.march(g, rays, tau, prec)
        if gi == 0:
            # each kernel once on the group's first block (module loading,
            # first-use setup), into a scratch field
            scratch = torch.zeros(6 * pb.ncell, dtype=torch.float32, device=dev)
            first = RayGroup(g.b0, min(g.b0 + 1, g.b1), g.base, g.nray)
            for m, code in modes:
                if code is None:
                    pb.rates_surrogate(first, rays, tau, scratch, sur)
                else:
                    pb.rates(first, rays, tau, scratch, code)
            del scratch
        for m, code in modes:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(pb.stream)
            if code is None:
                pb.rates_surrogate(g, rays, tau, fields[m], sur, counters)
            else:
                pb.rates(g, rays, tau, fields[m], code)
            e1.record(pb.stream)
            e1.synchronize()
            t[m] += e0.elapsed_time(e1) / 1e3
    pb.check_device_error()
    out = {}
    for m, _ in modes:
        out[m] = {"s": t[m], "gamma_cells_per_s": pb.ncell / t[m], "rays_per_s": pb.nray / t[m],
                  "speedup_vs_exact_f64": t["exact_f64"] / t[m]}
    if sur is not None:
        c = counters.cpu().numpy()
        out["surrogate"]["rays_surrogate"] = int(c[0])
        out["surrogate"]["rays_exact_fallback"] = int(c[1])
        out["surrogate"]["fallback_frac"] = float(c[1] / max(1, c[0] + c[1]))
    return out


# ------------------------------------------------------------ parity check
def sampled_parity(pb, wl, sur, runs: int = 16, length: int = 16, seed: int = 11):
    """The checker on this workload: seeded runs of target cells computed by
    the reference's own group loop (ARGOT's C, O1) and by the FP64 CPU
    oracle pipeline (FP64 march + FP64 rates) on O1's rays, against the
    device path on the target blocks holding them (oracle/sampled.py).
    Reported per rate mode: the largest relative error per output field
    over the sampled cells; for the reference-order path its ray lists and
    columns against O1 and its FP64 rates against O1's."""
    from argot_b200 import _lib as L
    from oracle.sampled import SampledParity, z_runs
    t0 = time.time()
    sp = SampledParity(wl, z_runs(wl.edge, runs, length, seed))
    ref, f64 = sp.reference(), sp.fp64()
    r64, rays = sp.device(pb, L.PRECISION_REFERENCE, L.RATE_EXACT_F64, want_rays=True)
    same_list, same_tau = sp.same_rays(rays)
    r32, rays_k = sp.device(pb, L.PRECISION_KAHAN, L.RATE_EXACT_F32, want_rays=True)
    out = {"sample": (f"{runs} seeded runs of {length} consecutive target cells along z "
                      f"({len(sp.all_cells())} cells, {len(ref['tgt'])} rays)"),
           "oracle": "O1 = ARGOT's C (reference order, FP32 march, FP64 rates); "
                     "FP64 = orc_march_f64 + orc_photoion_f64 on O1's rays",
           "reference_order": {"ray_lists_equal_O1": bool(same_list), "columns_bitwise_O1": bool(same_tau),
                               "exact_f64_rates_vs_O1": sp.rate_errors(r64, ref["rates"])},
           "kahan_columns_vs_fp64": sp.column_error_vs_f64(rays_k),
           "exact_f32_vs_fp64": sp.rate_errors(r32, f64["rates"])}
    if sur is not None:
        rs, _ = sp.device(pb, L.PRECISION_KAHAN, surrogate=sur)
        out["surrogate_vs_fp64"] = sp.rate_errors(rs, f64["rates"])
    out["s"] = time.time() - t0
    return out


# ------------------------------------------------------------ our arm
def run_ours(args):
    import torch
    from argot_b200 import _lib as L
    from argot_b200.pipeline import Problem

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    init_dist(ws, "nccl")
    dev = torch.device("cuda", local)
    sharded = args.shard and ws > 1
    # sharded: every rank holds the same problem and takes its own target slabs
    wl = make_workload(args.config, 0 if sharded else rank)
    prec = L.PRECISION_KAHAN if args.precision == "kahan" else L.PRECISION_REFERENCE
    mode = {"f32": L.RATE_EXACT_F32, "f64": L.RATE_EXACT_F64, "surrogate": L.RATE_SURROGATE}[args.rate]

    free, _ = torch.cuda.mem_get_info(dev)
    pb = Problem(wl, dev, max_group_rays=None)
    part, cell_ranges = (0, pb.nblocks), None
    if sharded:
        from argot_b200 import shard
        parts = shard.partition(pb.blk_count.cpu().numpy(), ws, wl.edge)
        cell_ranges = [shard.cells_of(b0, b1, wl.edge) for b0, b1 in parts]
        part = parts[rank]
    nray_mine = int(pb.blk_off_host[part[1]] - pb.blk_off_host[part[0]])
    ncell_mine = (cell_ranges[rank][1] - cell_ranges[rank][0]) if sharded else pb.ncell
    use_sur = mode == L.RATE_SURROGATE or not args.no_rate_modes
    per_ray = 16 + (28 if use_sur else 0)  # rays + columns (+ surrogate workspace)
    need = nray_mine * per_ray + (2 << 30)
    pb.restrict(*part, max_rays=int(free * 0.8 / per_ray) if need > free * 0.9 else None)
    stream = pb.stream
    rays, tau = pb.alloc_group_buffers()
    rates6 = torch.zeros(6 * pb.ncell, dtype=torch.float32, device=dev)
    single = len(pb.groups) == 1
    if single:
        pb.emit(pb.groups[0], rays)
    crossings = torch.zeros(1, dtype=torch.int64, device=dev)
    sur = load_surrogate(pb) if use_sur else None
    if mode == L.RATE_SURROGATE and sur is None:
        raise SystemExit("--rate surrogate needs trained weights (python -m argot_b200.train_surrogate)")

    def rate_pass(g):
        if mode == L.RATE_SURROGATE:
            pb.rates_surrogate(g, rays, tau, rates6, sur)
        else:
            pb.rates(g, rays, tau, rates6, mode)

    overlap = args.overlap if (single and mode != L.RATE_SURROGATE) else 0

    def step(count=None):
        if overlap > 1:
            # march of part p+1 on one stream, rates of part p on another
            pb.run(prec, mode, rates6, (rays, tau), count, keep_rays=True, overlap=overlap)
        else:
            for g in pb.groups:
                if not single:
                    pb.emit(g, rays)
                pb.march(g, rays, tau, prec, count)
                rate_pass(g)
        if sharded:  # the exchange step: every rank's rate slab to every rank
            shard.gather_rates(rates6, cell_ranges)

    # warm-up (the first one also counts the crossings)
    for w in range(args.warmup):
        step(crossings if w == 0 else None)
    torch.cuda.synchronize()
    pb.check_device_error()
    n_cross = int(crossings.item())

    # per-kernel split (one extra pass, events around each kernel)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    for g in pb.groups:
        if not single:
            pb.emit(g, rays)
        pb.march(g, rays, tau, prec)
    ev[1].record(stream)
    for g in pb.groups:
        rate_pass(g)
    ev[2].record(stream)
    torch.cuda.synchronize()
    t_march = ev[0].elapsed_time(ev[1]) / 1e3
    t_rates = ev[1].elapsed_time(ev[2]) / 1e3
    rate_modes = None if args.no_rate_modes else compare_rate_modes(pb, rays, tau, prec, sur)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = sampled_parity(pb, wl, sur)
        if rate_modes is not None:
            rate_modes["exact_f64"]["max_rel_err_vs_O1"] = parity["reference_order"]["exact_f64_rates_vs_O1"]
            rate_modes["exact_f32"]["max_rel_err_vs_fp64_oracle"] = parity["exact_f32_vs_fp64"]
            if "surrogate" in rate_modes and "surrogate_vs_fp64" in parity:
                rate_modes["surrogate"]["max_rel_err_vs_fp64_oracle"] = parity["surrogate_vs_fp64"]
    # the next stage of an iteration: the 27-point smoothing of the rates
    # (smooth_photoion_rate.c), on the device
    smoothed = torch.empty_like(rates6)
    pb.smooth(rates6, smoothed)
    es0, es1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    es0.record(stream)
    pb.smooth(rates6, smoothed)
    es1.record(stream)
    torch.cuda.synchronize()
    t_smooth = es0.elapsed_time(es1) / 1e3
    del smoothed

    clocks = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    pb.check_device_error()
    t_local = e0.elapsed_time(e1) / 1e3
    t = allmax(ws, t_local, dev)
    total_cross = allsum(ws, float(n_cross) * args.steps, dev)
    total_cells = allsum(ws, float(ncell_mine) * args.steps, dev)

    hbm, bf16, peak_kind = measured_peaks()
    alg_bytes = 16.0 * n_cross + 36.0 * nray_mine
    achieved = alg_bytes / t_march / 1e9
    launches_per_step = (2 * pb.part_count(overlap) if overlap > 1
                         else len(pb.groups) * (2 + (0 if single else 1)))

    # end to end through the C ABI from pinned host buffers (the timed
    # pass's buffers are released first: the e2e pass allocates its own)
    del rays, tau
    pb._sur_work = None
    torch.cuda.empty_cache()
    e2e = None if args.no_e2e else run_e2e(wl, dev, prec, mode, steps=max(1, min(args.steps, 3)),
                                           overlap=args.overlap,
                                           part=part if sharded else None, cell_ranges=cell_ranges)
    if e2e is not None and ws > 1:
        e2e["value"] = allsum(ws, e2e.pop("_crossings"), dev) / allmax(ws, e2e["s_per_step"], dev)
    elif e2e is not None:
        e2e.pop("_crossings")

    line = {
        "metric": METRIC, "value": total_cross / t, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded lognormal mesh + clustered sources)",
        "config": workload_config(wl, ws, sharded),
        "run": {"rays": nray_mine, "crossings": n_cross, "march": args.precision, "rates": args.rate,
                "ray_groups": len(pb.groups), "overlap_parts": overlap},
        "gamma_cells_per_s": total_cells / t,
        "split": {"march_s": t_march, "rates_s": t_rates,
                  "march_crossings_per_s": n_cross / t_march,
                  "rates_gamma_cells_per_s": ncell_mine / t_rates,
                  "rates_rays_per_s": nray_mine / t_rates,
                  "smooth_s": t_smooth, "smooth_gb_per_s": 2 * 24 * pb.ncell / t_smooth / 1e9},
        "roofline": {"kernel": "k_march_rays", "bound": "hbm", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": f"{peak_kind} hbm_gbs",
                     "traffic": MARCH_DRAM_BYTES_PER_CROSSING * n_cross,
                     "l2_traffic": MARCH_L2_BYTES_PER_CROSSING * n_cross,
                     "traffic_source": (f"ncu DRAM bytes per crossing on 256^3 / 16 sources "
                                        f"({MARCH_DRAM_BYTES_PER_CROSSING} B; L2 {MARCH_L2_BYTES_PER_CROSSING} B), "
                                        f"scaled by this launch's crossings"),
                     "dram_gbs": MARCH_DRAM_BYTES_PER_CROSSING * n_cross / t_march / 1e9,
                     "dram_frac": MARCH_DRAM_BYTES_PER_CROSSING * n_cross / t_march / 1e9 / hbm,
                     "limiter": ("latency of the L1/L2-hit gathers (ncu: long-scoreboard stalls 14.1 per issue, "
                                 "issue active 60%); DRAM moves 2.0 B and L2 serves 6.8 B of the 16 B per "
                                 "crossing that the bytes model counts"),
                     "algorithmic_bytes": alg_bytes,
                     "bytes_model": "16 B per crossing + 36 B per ray"},
        "clocks": clk,
        "gpu_launches": launches_per_step * args.steps,
    }
    if rate_modes is not None:
        line["rate_modes"] = rate_modes
    if parity is not None:
        line["parity"] = parity
    if e2e is not None:
        line["e2e"] = e2e
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_sample(wl, target_seconds=args.cpu_seconds, R=reference_setup(wl))
            cb.pop("_probe_rays", None)
            line["cpu_baseline"] = cb
        except Exception as exc:  # the baseline must not hide our own number
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                    "kind": "reference", "sample": f"failed: {exc}"}
    pb.close()
    if rank == 0 and ws == 1 and not args.no_reference_gpu:
        torch.cuda.empty_cache()
        try:
            line["reference_gpu"] = reference_gpu_sample(wl, target_rays=args.reference_gpu_rays)
        except Exception as exc:  # the baseline must not hide our own number
            line["reference_gpu"] = {"value": None, "unit": UNIT, "kind": "reference",
                                     "sample": f"failed: {exc}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_e2e(wl, dev, prec, mode, steps=2, part=None, cell_ranges=None, overlap=0):
    """Same metric through the public C ABI with host buffers: each step
    copies the mesh fields and the source table from pinned host memory,
    builds the tree, generates the rays on the device, marches, computes the
    rates and copies the six rate fields back to pinned host memory.  With
    `part` (sharded ranks) only that block range is computed and the rate
    slabs are all-gathered before the copy back."""
    import torch
    from argot_b200 import _lib as L
    from argot_b200.pipeline import Problem
    pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in wl.fields()]
    out = torch.empty(6 * wl.ncell, dtype=torch.float32).pin_memory()
    h2d = sum(p.numel() * 4 for p in pin) + wl.nsrc * (12 + 8 + 8)
    times = []
    cross = None
    sur = None
    if mode == L.RATE_SURROGATE:
        from argot_b200 import surrogate as S
        sur = S.Surrogate.from_file()  # weights stay resident, like a solver's
    for s in range(steps + 1):  # first pass warms the caching allocator
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pb = Problem(wl, dev, host_fields=pin)
        if part is not None:
            pb.restrict(*part)
        if sur is not None:
            pb.set_blackbody()
        rays, tau = pb.alloc_group_buffers()
        rates6 = torch.zeros(6 * pb.ncell, dtype=torch.float32, device=dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        if sur is None and overlap > 1 and len(pb.groups) == 1:
            pb.run(prec, mode, rates6, (rays, tau), cnt, overlap=overlap)
        else:
            for g in pb.groups:
                pb.emit(g, rays)
                pb.march(g, rays, tau, prec, cnt)
                if sur is not None:
                    pb.rates_surrogate(g, rays, tau, rates6, sur)
                else:
                    pb.rates(g, rays, tau, rates6, mode)
        if part is not None:
            from argot_b200 import shard
            rates6 = shard.gather_rates(rates6, cell_ranges).view(-1)
        out.copy_(rates6, non_blocking=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        cross = int(cnt.item())
        pb.close()
        del rays, tau
        if s > 0:
            times.append(dt)
    t = statistics.median(times)
    return {"value": cross / t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(out.numel() * 4), "s_per_step": t, "_crossings": cross,
            "includes": "H2D fields, host tree, device ray generation, march, rates, D2H rates"}


# ------------------------------------------------------------ batched arm
def run_batched(args):
    """48 problems of uneven size (mesh edge from {32,48,64,96,128}, 4-512
    sources, sigma_ln in [0.5, 1.5]) per GPU; a step is one replay of the
    CUDA graph of the persistent batch launch (march + EXACT_F32 rates of
    every ray of every problem), configured by the autotuner first."""
    import torch
    from argot_b200.batch import Batch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    init_dist(ws, "nccl")
    dev = torch.device("cuda", local)
    wls = make_workload(args.config, rank)
    B = Batch(wls, dev)
    stream = torch.cuda.current_stream(dev)
    cfg, tune_ms = B.tune(reps=1)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    B.run(cnt)
    torch.cuda.synchronize()
    B.check_device_error()
    n_cross = int(cnt.item())
    for _ in range(args.warmup):
        B.graph_launch()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        B.graph_launch()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    B.check_device_error()
    t = allmax(ws, e0.elapsed_time(e1) / 1e3, dev)
    total_cross = allsum(ws, float(n_cross) * args.steps, dev)
    total_cells = allsum(ws, float(B.ncell) * args.steps, dev)
    hbm, _, peak_kind = measured_peaks()
    alg_bytes = 16.0 * n_cross + 24.0 * B.nray
    achieved = alg_bytes / (t / args.steps) / 1e9 if ws == 1 else None
    e2e = None if args.no_e2e else batched_e2e(B, wls, dev, steps=max(1, min(args.steps, 3)))
    if e2e is not None:
        cross = e2e.pop("_crossings")
        e2e["value"] = allsum(ws, cross, dev) / allmax(ws, e2e["s_per_step"], dev)
    line = {
        "metric": METRIC, "value": total_cross / t, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lognormal meshes + uniform sources)",
        "config": {"workload": f"{args.config}: {len(wls)} problems, edges "
                               f"{sorted(set(w.edge for w in wls))}, sources "
                               f"{min(w.nsrc for w in wls)}-{max(w.nsrc for w in wls)}",
                   "rays": B.nray, "crossings": n_cross, "cells": B.ncell,
                   "launch": "one persistent kernel per step, replayed as a CUDA graph",
                   "autotuned": cfg, "tune_best_ms": tune_ms,
                   "l2": f"inputs larger than L2 ({B.nray * 4 / 1e9:.1f} GB rays); no flush",
                   "parallelism": f"{ws} independent batches (one per GPU)"},
        "gamma_cells_per_s": total_cells / t,
        "roofline": {"kernel": "k_batch (march + rates fused)", "bound": "hbm", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm if achieved else None,
                     "peak_kind": f"{peak_kind} hbm_gbs", "traffic": None,
                     "algorithmic_bytes": alg_bytes,
                     "bytes_model": "16 B per crossing + 24 B per ray (end points; columns stay on chip)"},
        "clocks": clk,
        "gpu_launches": args.steps,
    }
    if e2e is not None:
        line["e2e"] = e2e
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            big = max(wls, key=lambda w: (w.edge, w.nsrc))
            cb = cpu_sample(big, target_seconds=args.cpu_seconds, R=reference_setup(big))
            cb.pop("_probe_rays", None)
            cb["sample"] = f"largest problem of the batch ({big.name}): " + cb["sample"]
            line["cpu_baseline"] = cb
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                    "kind": "reference", "sample": f"failed: {exc}"}
    B.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batched_e2e(B, wls, dev, steps=2):
    """The batch step through the public C ABI with host buffers: every
    problem's four fields copied from pinned host memory and packed, the
    batch graph replayed, every problem's six rate fields copied back to
    pinned host memory.  The trees and rays are set up once (they depend
    only on the source positions and the mesh geometry)."""
    import torch
    pins = [[torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in wl.fields()] for wl in wls]
    outs = [torch.empty(6 * wl.ncell, dtype=torch.float32).pin_memory() for wl in wls]
    h2d = sum(p.numel() * 4 for ps in pins for p in ps)
    d2h = sum(o.numel() * 4 for o in outs)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    times = []
    for s in range(steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for pb, ps in zip(B.problems, pins):
            for dst, src in zip(pb.fields, ps):
                dst.copy_(src, non_blocking=True)
            pb.pack()
        if s == 0:
            B.run(cnt)
        else:
            B.graph_launch()
        for o, r in zip(outs, B.rates):
            o.copy_(r, non_blocking=True)
        torch.cuda.synchronize()
        if s > 0:
            times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    cross = int(cnt.item())
    return {"value": cross / t, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "s_per_step": t, "_crossings": cross,
            "includes": "H2D fields + pack of every problem, batch graph replay, D2H rates"}


# ------------------------------------------------------------ ART
def art_fields(wl):
    """The eight input planes of the diffuse-radiation path from a
    workload's mesh: dens, fHI, fHII, fHeI, fHeII, fHeIII, felec, uene, with
    fHII = 1 - fHI, fHeIII = 1 - fHeI - fHeII, the electrons of both, and a
    temperature of 100 K in neutral gas rising to 2e4 K with fHII (uene in
    units where T = uene * ART_UENETOK * wmol, as run_param.uenetok)."""
    helium_fact = 0.0811258278  # prim_chem/chemistry.h:25
    dens, fhi, fhei, fheii = [np.asarray(a, np.float64) for a in wl.fields()]
    fhii = 1.0 - fhi
    fheiii = np.clip(1.0 - fhei - fheii, 0.0, 1.0)
    felec = fhii + helium_fact * (fheii + 2.0 * fheiii)
    temp = 100.0 + (2.0e4 - 100.0) * fhii
    wmol = 1.0 / ((1.0 + felec) * 0.755 + 0.25 * 0.245)
    uene = temp / (ART_UENETOK * wmol)
    return np.stack([dens, fhi, fhii, fhei, fheii, fheiii, felec, uene]).astype(np.float32)


def art_reference(wl, planes, threads=None):
    """ARGOT's own CPU calc_diffuse_photon_radiation (OpenMP over all host
    cores) on the same mesh: (wall seconds, rates)"""
    from oracle.oracle import RefLib
    R = RefLib(wl.edge)
    R.init(wl.lunit, wl.denstonh, wl.theta, threads or os.cpu_count() or 1)
    R.art_init(ART_UENETOK)
    R.art_set_mesh(planes)
    rates, t = R.art_run()
    return t, rates


def run_art(args):
    """The ART diffuse-radiation path (argot_b200_art_rates, all 768
    directions) on one GPU: K timed passes with the fields resident, CUDA
    events; e2e through the same call from pinned host buffers."""
    import torch
    from argot_b200 import _lib as L
    from argot_b200 import diffuse as D
    from argot_b200.pipeline import unit_box_grid
    ws, rank, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    init_dist(ws, "nccl")
    wl = make_workload(args.config, rank)
    planes = art_fields(wl)
    g = unit_box_grid(wl.edge, wl.lunit, wl.denstonh)
    n = wl.ncell
    f = torch.from_numpy(planes).to(dev)
    rates = torch.zeros(6 * n, dtype=torch.float32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    art = D.Diffuse()
    apass = art.default_pass(g)
    stream = torch.cuda.current_stream(dev)
    lib = L.load()

    def step(count=None):
        art.rates(g, ART_UENETOK, f, rates, angles_per_pass=apass, crossings=count, stream=stream.cuda_stream)

    for w in range(args.warmup):
        step(cnt if w == 0 else None)
    torch.cuda.synchronize()
    L.check(lib.argot_b200_check_device_error(stream.cuda_stream), "device error")
    steps_per_pass = int(cnt.item())
    clocks = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    t = allmax(ws, e0.elapsed_time(e1) / 1e3, dev)
    total = allsum(ws, float(steps_per_pass) * args.steps, dev)
    hbm, _, peak_kind = measured_peaks()
    # algorithmic bytes of one pass: per step two float4 of cell data read
    # and one float4 reduction; per cell and direction one float4 folded;
    # per cell 8 planes in, 6 planes of totals and 6 rate planes
    alg = 48.0 * steps_per_pass + 16.0 * n * art.nang + 4.0 * n * (8 + 6 + 12)
    achieved = alg / (t / args.steps) / 1e9
    # e2e: the 8 planes from pinned host memory, the pass, the rates back
    pin_f = torch.from_numpy(planes).pin_memory()
    out = torch.empty(6 * n, dtype=torch.float32).pin_memory()
    times = []
    for s_ in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f.copy_(pin_f, non_blocking=True)
        rates.zero_()
        step()
        out.copy_(rates, non_blocking=True)
        torch.cuda.synchronize()
        if s_ > 0:
            times.append(time.perf_counter() - t0)
    te = statistics.median(times)
    got = out.view(6, -1).numpy().copy()
    art.close()
    line = {
        "metric": ART_METRIC, "value": total / t, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lognormal mesh, ionisation around clustered sources)",
        "config": {"workload": f"art on {wl.name}", "mesh": f"{wl.edge}^3", "directions": art.nang,
                   "angles_per_pass": apass, "steps_per_pass": steps_per_pass,
                   "l2": "cell data 1 GB at 256^3, 67 MB at 128^3; accumulators larger than L2; no flush",
                   "parallelism": f"{ws} independent meshes (one per GPU)"},
        "roofline": {"kernel": "k_art_cells + k_art_trace + k_art_fold (one pass)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": f"{peak_kind} hbm_gbs", "traffic": None,
                     "bytes_model": "48 B per ray-cell step + 16 B per cell and direction + 104 B per cell"},
        "e2e": {"value": float(steps_per_pass) / te, "unit": UNIT, "h2d_bytes_per_step": int(planes.nbytes),
                "d2h_bytes_per_step": int(6 * n * 4), "s_per_step": te},
        "clocks": clk,
        "gpu_launches": (2 + 2 * ((art.nang + apass - 1) // apass)) * args.steps,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            tr, ref = art_reference(wl, planes)
            rel = np.abs(got.astype(np.float64) - ref) / np.maximum(np.abs(ref.astype(np.float64)), 1e-300)
            big = np.abs(ref) > 1e-6 * np.abs(ref).max(axis=1, keepdims=True)
            line["cpu_baseline"] = {"value": steps_per_pass / tr, "unit": UNIT, "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"one whole ART pass on the same {wl.edge}^3 mesh, {tr:.1f} s"}
            line["max_rel_err_vs_reference"] = float(rel[big].max())
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"failed: {exc}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ------------------------------------------------------------ reference arm
def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    wl = make_workload(args.config, 0)
    if isinstance(wl, list):  # a batch: the largest problem stands for it
        wl = max(wl, key=lambda w: (w.edge, w.nsrc))
    R = reference_setup(wl)
    vals, walls = [], []
    info = None
    for s in range(args.warmup + args.steps):
        r = cpu_sample(wl, target_seconds=args.ref_seconds, R=R, seed=s)
        if s >= args.warmup:
            vals.append(r["value"])
            walls.append(r["wall_s"])
            info = r
    v = statistics.median(vals)
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(walls),
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic (seeded lognormal mesh + clustered sources)",
        "config": workload_config(wl, ws, False),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "reference",
                         "sample": info["sample"] + " (per step; median over steps)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_art(args):
    """the reference's CPU ART on the same mesh, one whole pass per step"""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle.oracle import RefLib
    wl = make_workload(args.config, 0)
    planes = art_fields(wl)
    R = RefLib(wl.edge)
    R.init(wl.lunit, wl.denstonh, wl.theta, os.cpu_count() or 1)
    R.art_init(ART_UENETOK)
    R.art_set_mesh(planes)
    ts = []
    for s in range(args.warmup + args.steps):
        _, t = R.art_run()
        if s >= args.warmup:
            ts.append(t)
    t = statistics.median(ts)
    steps = art_step_count(wl)
    v = steps / t
    print(json.dumps({
        "metric": ART_METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "impl": "reference", "data": "synthetic (seeded lognormal mesh)",
        "config": {"workload": f"art on {wl.name}", "mesh": f"{wl.edge}^3"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"whole ART passes, median {t:.1f} s"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def art_step_count(wl):
    """ray-cell steps of one ART pass (the reference's float DDA gives the
    same cells): counted by the GPU kernel when one is present, else by a
    NumPy walk of every ray"""
    import torch
    if torch.cuda.is_available():
        from argot_b200 import diffuse as D
        from argot_b200.pipeline import unit_box_grid
        g = unit_box_grid(wl.edge, wl.lunit, wl.denstonh)
        f = torch.from_numpy(art_fields(wl)).cuda()
        r = torch.zeros(6 * wl.ncell, dtype=torch.float32, device="cuda")
        c = torch.zeros(1, dtype=torch.int64, device="cuda")
        art = D.Diffuse()
        art.rates(g, ART_UENETOK, f, r, crossings=c)
        torch.cuda.synchronize()
        art.close()
        return int(c.item())
    raise SystemExit("the ART step count needs the GPU kernel")


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__,
                                formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--config", choices=CONFIGS, default="largest")
    p.add_argument("--precision", choices=("kahan", "reference"), default="kahan")
    p.add_argument("--rate", choices=("f32", "f64", "surrogate"), default="f32")
    p.add_argument("--no-rate-modes", action="store_true",
                   help="skip the one-pass comparison of the three rate kernels")
    p.add_argument("--shard", action="store_true",
                   help="N>1: one problem, target slabs sharded over the ranks (strong scaling)")
    p.add_argument("--overlap", type=int, default=32,
                   help="cut the ray group into N parts and overlap the march of one part with the "
                        "rates of the previous one on two streams (0: one stream, kernels in sequence)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-parity", action="store_true",
                   help="skip the sampled parity check against the reference and the FP64 oracle")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="skip the sample of ARGOT's own GPU kernels built for sm_100a")
    p.add_argument("--reference-gpu-only", action="store_true",
                   help="run only the reference-GPU sample of the config and print it (a profiling case)")
    p.add_argument("--reference-gpu-rays", type=int, default=2_000_000,
                   help="rays in the reference-GPU sample")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--ref-seconds", type=float, default=15.0)
    args = p.parse_args(argv)
    if args.reference_gpu_only:
        wl = make_workload(args.config, 0)
        if isinstance(wl, list):
            wl = max(wl, key=lambda w: (w.edge, w.nsrc))
        print(json.dumps({"config": wl.name,
                          "reference_gpu": reference_gpu_sample(wl, target_rays=args.reference_gpu_rays)}),
              flush=True)
    elif args.impl == "reference" and args.config.startswith("art"):
        run_reference_art(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config.startswith("art"):
        run_art(args)
    elif args.config.startswith("batched"):
        run_batched(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
