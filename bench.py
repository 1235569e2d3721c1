#!/usr/bin/env python
"""Projector-pair throughput on B200: cone-beam 256^3 -> 360 x 512^2.

One step = the forward projection of all 360 views of a 256^3 FP32 volume
(closed-form cubic B-spline footprint, SID 1000 mm, SDD 1500 mm, 1 mm
voxels and detector cells) followed by the transpose of all 360 views: the
data-fidelity operator pair of one reconstruction iteration.  The metric
counts each per-view forward and each per-view transpose as one projection
(views * 2 per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) every rank projects its own 360-view scan (views
are independent units, weak scaling, no data-path collective); the timing
is the maximum over ranks.  Rank 0 prints one JSON line.

``--impl reference`` times the reference plugin C (compiled from its
sources into oracle/_ref, FP64, single-threaded per call) on the host
cores, views spread over all available threads, on a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
ND = 512
VIEWS = 360
SID, SDD = 1000.0, 1500.0
WORKLOAD = (f"cone-beam circular orbit, {N}^3 FP32 volume of 20 random ellipsoids -> "
            f"{VIEWS} x {ND}x{ND} detector, 1 mm voxels/cells, SID {SID:g} mm, SDD {SDD:g} mm, "
            "closed-form cubic B-spline footprint; step = forward + transpose of all views")


def _env_int(name, default):
    v = os.environ.get(name)
    return int(v) if v is not None else default


def scan(rank=0, views=VIEWS):
    from yoricktrtt_b200 import geometry as G
    theta0 = rank * (2 * math.pi / views) / max(1, _env_int("WORLD_SIZE", 1))
    th = theta0 + np.arange(views) * (2 * math.pi / views)
    return G.circular_scan_3d(N, N, N, 1.0, 3, ND, ND, 1.0, 1.0, views,
                              mode=G.TRTT_CONE_BEAM, rsc=SID, rsd=SDD, theta=th)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference plugin (or the oracle port) on host threads
# ---------------------------------------------------------------------------
_CPU_INPUTS = []


def _cpu_inputs():
    """Scan, FP64 phantom and one detector image of the workload (built once)."""
    if not _CPU_INPUTS:
        from yoricktrtt_b200 import phantoms as P
        _CPU_INPUTS.extend([scan(0, VIEWS),
                            np.ascontiguousarray(P.ellipsoids_3d(N, N, N, n=20, seed=0,
                                                                 dtype=np.float64)),
                            np.ascontiguousarray(np.random.default_rng(0).random((ND, ND)))])
    return _CPU_INPUTS


def cpu_pair_sample(nviews_sample, threads=None):
    """Time nviews_sample forward+transpose view pairs of the workload with the
    reference C on `threads` host threads (views spread over threads, private
    outputs, as the reference's MPY decomposition does).  Returns
    (projections/s, seconds, kind, threads)."""
    from oracle import oracle
    kind = "reference" if oracle.ref_available() else "port"
    orc = oracle.get("ref" if kind == "reference" else "port")
    sc, vol, det_in = _cpu_inputs()
    threads = threads or (os.cpu_count() or 1)
    threads = max(1, min(threads, nviews_sample))
    views = np.linspace(0, VIEWS - 1, nviews_sample).astype(int)

    def work(vs):
        out = np.zeros((ND, ND))  # private outputs, one pair per thread
        back = np.zeros_like(vol)
        for v in vs:
            out.fill(0.0)
            orc.cb3d(out, vol, sc, int(v), 0)
            back.fill(0.0)
            orc.cb3d(back, det_in, sc, int(v), 1)

    chunks = [views[t::threads] for t in range(threads)]
    t0 = time.perf_counter()
    ths = [threading.Thread(target=work, args=(c,)) for c in chunks]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    return 2 * nviews_sample / dt, dt, kind, threads


def _host_cores():
    if hasattr(os, "sched_getaffinity"):
        return len(os.sched_getaffinity(0))
    return os.cpu_count() or 1


def cpu_baseline_measure(warmup=1, steps=2):
    """The CPU baseline as both arms report it: one forward + transpose view
    pair per host thread and step (at most 256 threads: each holds a private
    FP64 output volume of 134 MB), `warmup` untimed steps, the median of
    `steps` timed ones."""
    cores = _host_cores()
    sample = max(1, min(cores, VIEWS, 256))
    times = []
    kind = thr = None
    for it in range(warmup + steps):
        _, dt, kind, thr = cpu_pair_sample(sample, cores)
        if it >= warmup:
            times.append(dt)
    dt = statistics.median(times)
    return {"value": 2 * sample / dt, "unit": "projections/s", "cores": thr, "kind": kind,
            "sample": f"{sample} view pairs (forward + transpose) of the workload per step, one per "
                      f"host thread, reference C in FP64; {warmup} warm-up + median of {steps} steps",
            "pairs_per_step": sample, "seconds_per_step": dt}


def run_reference(args):
    rank = _env_int("RANK", 0)
    if rank != 0:
        return 0
    try:
        from oracle import oracle
        oracle.build(ref=True)
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"oracle build failed: {e}"}))
        return 0
    cpu = cpu_baseline_measure(warmup=args.warmup, steps=args.steps)
    value, sample, dt = cpu["value"], cpu["pairs_per_step"], cpu["seconds_per_step"]
    line = {
        "impl": "reference", "metric": "fwd+back projections/s", "value": value,
        "unit": "projections/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{sample} of {VIEWS} view pairs per step"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "projections/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
# names of the kernels the step launches (per direction), for the roofline:
# the group kernels when the scan's views group by turns of the grid, else
# the per-view kernels
KERNELS = {True: ("k_fwd3d_group (direct, view groups x detector-row bands)",
                  "k_back3d_group (transpose, column orbits)"),
           False: ("k_fwd3d_band_fast (direct, detector-row bands)",
                   "k_back3d_col_fast (transpose, column gather)")}
PARITY_VIEWS = (0, 137, 271)


def _counters():
    """ncu counters of the two kernels at this workload, committed under
    profiles/ (DRAM traffic and executed warp instructions per launch)."""
    try:
        with open(os.path.join(ROOT, "profiles", "counters_cone256.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def timed_pairs(pr, x, sino, back, flush, steps, warmup, world, barrier):
    """`warmup` untimed then `steps` timed forward + transpose pairs; returns
    (total ms, per-step forward ms, per-step transpose ms, launches)."""
    import torch
    from yoricktrtt_b200 import _lib
    stream = torch.cuda.current_stream()

    def step(ev=None):
        sino.zero_()
        back.zero_()
        if ev:
            ev[0].record(stream)
        pr.forward(x, out=sino, layout="columns")
        if ev:
            ev[1].record(stream)
        pr.backward(sino, out=back, layout="columns")
        if ev:
            ev[2].record(stream)
        flush.fill_(1.0)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    pr.status()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = _lib.launch_count()
    barrier()
    t_start.record(stream)
    for k in range(steps):
        step(evs[k])
    t_end.record(stream)
    barrier()
    launches = _lib.launch_count() - launches0
    pr.status()
    return (t_start.elapsed_time(t_end), [e[0].elapsed_time(e[1]) for e in evs],
            [e[1].elapsed_time(e[2]) for e in evs], launches)


def parity_block(pr, sc, vol_h, sino):
    """Relative L2 of the timed forward output on sampled views against the
    FP64 reference C, and of the transpose of those views of the timed output
    (one full 360-view transpose launch, the other views zero) against the
    reference's sum over them.  Runs outside the timed region."""
    import concurrent.futures as cf
    import torch
    from oracle import oracle
    kind = "ref" if oracle.ref_available() else "port"
    orc = oracle.get(kind)
    vol64 = np.ascontiguousarray(vol_h, dtype=np.float64)
    views = list(PARITY_VIEWS)
    got = {v: sino[v].double().cpu().numpy() for v in views}
    y = torch.zeros_like(sino)
    for v in views:
        y[v] = sino[v]
    b = pr.backward(y, layout="xyz").double().cpu().numpy()
    pr.status()

    def fwd(v):
        out = np.zeros((ND, ND))
        orc.cb3d(out, vol64, sc, v, 0)
        return out

    def bwd(v):
        out = np.zeros((N, N, N))
        orc.cb3d(out, np.ascontiguousarray(got[v]), sc, v, 1)
        return out

    with cf.ThreadPoolExecutor(max(1, min(2 * len(views), _host_cores()))) as ex:
        fr = list(ex.map(fwd, views))
        br = list(ex.map(bwd, views))
    ferr = [float(np.linalg.norm(got[v] - r) / np.linalg.norm(r)) for v, r in zip(views, fr)]
    ref_b = sum(br)
    berr = float(np.linalg.norm(b - ref_b) / np.linalg.norm(ref_b))
    return {"views": views, "forward_rel_l2": ferr, "transpose_rel_l2": berr,
            "max_rel_l2": max(ferr + [berr]), "bar": 1e-5,
            "oracle": ("reference C compiled from its sources, FP64" if kind == "ref"
                       else "FP64 C restatement (bit-identical to the reference C)")}


def run_dropin_e2e(sc, vol_h, nsample=8):
    """The per-view plugin path a Yorick closure takes: one trtt_CB3D_cubic
    call per view and direction on host FP64 arrays (pageable, as Yorick's
    are), accumulating into `out`; `nsample` view pairs, scaled."""
    from yoricktrtt_b200 import dropin
    vol64 = np.ascontiguousarray(vol_h, dtype=np.float64)
    out = np.zeros((ND, ND))
    back = np.zeros((N, N, N))
    views = np.linspace(0, VIEWS - 1, nsample + 1).astype(int)

    def pair(v):
        out.fill(0.0)
        dropin.scan3d_call("CB3D", out, vol64, sc, int(v), 0)
        dropin.scan3d_call("CB3D", back, out, sc, int(v), 1)

    pair(views[0])  # warm-up
    t0 = time.perf_counter()
    for v in views[1:]:
        pair(v)
    dt = (time.perf_counter() - t0) / nsample
    nvox, npix = N ** 3, ND * ND
    return {"value": 2 / dt, "unit": "projections/s", "ms_per_view_pair": dt * 1e3,
            "path": "trtt_CB3D_cubic per view and direction (the symbol the Yorick closure "
                    "_trtt_single_3D_projector calls), pageable host FP64 arrays, out += H in",
            "sample": f"{nsample} view pairs of the workload, per-pair time scaled to the rate",
            # direct: the FP64 volume up, the image (accumulated) up and
            # down; transpose: the FP64 image up, the volume's FP32
            # contribution down (added into the host volume on the host)
            "h2d_bytes_per_view_pair": 8 * (nvox + npix) + 8 * npix,
            "d2h_bytes_per_view_pair": 8 * npix + 4 * nvox}


def run_b200(args):
    import torch
    import torch.distributed as dist
    from yoricktrtt_b200 import phantoms as P
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    sc = scan(rank)
    pr = Projector3D(sc)
    if args.band_rows or args.warps:
        pr.set_tiles(args.band_rows, args.warps)
    if args.no_symmetry:
        pr.set_symmetry(False)
    vol_h = P.ellipsoids_3d(N, N, N, n=20, seed=0, dtype=np.float32)
    x = columns_from_xyz(torch.tensor(vol_h, device=dev))
    sino = torch.zeros(VIEWS, ND, ND, device=dev)
    back = torch.zeros_like(x)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if world > 1:
            t = torch.tensor([v], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            v = float(t.item())
        return v

    with ClockSampler(local) as clk:
        ms, fwd_ms, back_ms, launches = timed_pairs(pr, x, sino, back, flush, args.steps,
                                                    args.warmup, world, barrier)
    ms = max_over_ranks(ms)
    total_proj = 2 * VIEWS * world * args.steps
    value = total_proj / (ms / 1e3)
    fwd_avg, back_avg = statistics.mean(fwd_ms), statistics.mean(back_ms)
    clocks = clk.summary()

    # parity of the timed output (rank 0, outside the timed region)
    parity = None
    if rank == 0 and not args.skip_parity:
        parity = parity_block(pr, sc, vol_h, sino)
    barrier()

    # the same pair with the per-view kernels (no footprint sharing between
    # views related by turns of the grid), for comparison
    per_view = None
    if not args.skip_dense and not args.no_symmetry and sum(pr.groups()[1:]) > 0:
        pr.set_symmetry(False)
        psteps = max(1, min(args.steps, 2))
        pms, pfwd, pback, _ = timed_pairs(pr, x, sino, back, flush, psteps, 1, world, barrier)
        pms = max_over_ranks(pms)
        per_view = {"value": 2 * VIEWS * world * psteps / (pms / 1e3), "unit": "projections/s",
                    "fwd_ms": statistics.mean(pfwd), "back_ms": statistics.mean(pback),
                    "steps": psteps, "kernels": "k_fwd3d_band_fast + k_back3d_col_fast"}
        pr.set_symmetry(True)  # back to the default group kernels

    # the same pair on a dense volume (every voxel non-zero, as a
    # reconstruction iterate is): no zero-voxel shortcut applies
    dense = None
    if not args.skip_dense:
        rng = np.random.default_rng(1)
        vd = (vol_h + 0.05 + 0.1 * rng.random(vol_h.shape)).astype(np.float32)
        xd = columns_from_xyz(torch.tensor(vd, device=dev))
        dsteps = max(1, min(args.steps, 3))
        dms, dfwd, dback, _ = timed_pairs(pr, xd, sino, back, flush, dsteps, 1, world, barrier)
        dms = max_over_ranks(dms)
        dense = {"value": 2 * VIEWS * world * dsteps / (dms / 1e3), "unit": "projections/s",
                 "ms_per_step": dms / dsteps, "fwd_ms": statistics.mean(dfwd),
                 "back_ms": statistics.mean(dback), "steps": dsteps,
                 "volume": "the phantom + 0.05 + U[0, 0.1): every voxel non-zero"}
        del xd

    # the same pair with the tabulated footprint (10 001 samples of the cubic
    # B-spline primitive, the reference's size_footprint): the table model
    # keeps the per-view kernels, whose table slots must be the reference's
    table_model = None
    if not args.skip_dense:
        from yoricktrtt_b200 import footprint as F
        from yoricktrtt_b200.projectors import Projector3D
        prt = Projector3D(sc, F.make_footprint(3, 10001))
        tsteps = 1
        tms, tfwd, tback, _ = timed_pairs(prt, x, sino, back, flush, tsteps, 1, world, barrier)
        tms = max_over_ranks(tms)
        table_model = {"value": 2 * VIEWS * world * tsteps / (tms / 1e3), "unit": "projections/s",
                       "fwd_ms": statistics.mean(tfwd), "back_ms": statistics.mean(tback),
                       "steps": tsteps, "footprint": "table of 10001 samples (FP64), per-view kernels",
                       "kernels": "k_fwd3d_band_table + k_back3d_col_fast (table model)"}
        prt.close()

    # roofline of the dominant kernel: algorithmic bytes per launch (per-view
    # streaming model: the forward reads the volume and writes one detector
    # image per view, the transpose reads one image and writes the volume
    # contribution per view) / measured launch duration; the kernels are
    # bound by instruction issue, reported beside it from the committed ncu
    # instruction counts of the same kernels at this workload
    nvox, npix = N ** 3, ND * ND
    grouped = pr.groups()[1] + pr.groups()[2] > 0 and not args.no_symmetry
    fwd_kernel, back_kernel = KERNELS[grouped]
    if back_avg >= fwd_avg:
        kern, kms = back_kernel, back_avg
    else:
        kern, kms = fwd_kernel, fwd_avg
    alg_bytes = VIEWS * (4 * nvox + 4 * npix)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg_bytes / (kms / 1e3) / 1e9
    counters = _counters()
    kc = counters.get("kernels", {}).get(kern.split()[0], {})
    traffic = kc.get("dram_bytes")
    issue = None
    if kc.get("warp_inst"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clocks.get("sm_mhz") or 1965.0
        slots = kms * 1e-3 * sms * 4 * mhz * 1e6  # one warp instruction per SMSP and cycle
        issue = {"warp_inst_per_launch": kc["warp_inst"],
                 "thread_inst_per_voxel_view": 32.0 * kc["warp_inst"] / (nvox * VIEWS),
                 "issue_frac": kc["warp_inst"] / slots,
                 "issue_active_pct_ncu": kc.get("issue_active_pct"),
                 "peak": f"{sms} SMs x 4 schedulers x 1 warp instruction per cycle at {mhz:g} MHz",
                 "source": "profiles/counters_cone256.json (" + counters.get("command", "ncu") + ")"}

    # end to end through the batched host-buffer C ABI on every rank at once
    # (each rank its own scan), whole-job rate over the slowest rank
    e2e = None
    if not args.skip_e2e:
        barrier()
        e2e = run_e2e(sc, vol_h, args, dev)
        e2e["ms_per_step"] = max_over_ranks(e2e["ms_per_step"])
        e2e["value"] = 2 * VIEWS * world / (e2e["ms_per_step"] / 1e3)
        e2e["h2d_bytes_per_step"] *= world  # all ranks
        e2e["d2h_bytes_per_step"] *= world
    dropin_e2e = None
    if rank == 0 and world == 1 and not args.skip_e2e:
        dropin_e2e = run_dropin_e2e(sc, vol_h)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        try:
            cpu = cpu_baseline_measure(warmup=1, steps=2)
        except Exception as e:  # pragma: no cover
            cpu = {"value": None, "unit": "projections/s", "cores": 0, "kind": "port",
                   "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": "fwd+back projections/s", "value": value, "unit": "projections/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "views_per_gpu": VIEWS, "volume": [N, N, N],
                       "detector": [ND, ND], "footprint": "cubic",
                       "l2": "256 MiB buffer written between steps (inside the timed region); "
                             "the 360-view detector stack (377 MB) exceeds L2",
                       "fwd_ms": fwd_avg, "back_ms": back_avg,
                       "band_rows": args.band_rows or "auto",
                       "view_groups": {"singles": pr.groups()[0], "half_turn_pairs": pr.groups()[1],
                                       "quarter_turn_quads": pr.groups()[2],
                                       "used": bool(grouped)}},
            "parity": parity,
            "dense": dense,
            "table_model": table_model,
            "per_view_kernels": per_view,
            "roofline": {"bound": "issue", "kernel": kern, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                         "algorithmic_bytes_per_launch": alg_bytes, "issue": issue,
                         "note": "achieved/peak/frac: the HBM streaming model (not the binding "
                                 "limit); issue: executed warp instructions per launch over the "
                                 "launch's issue slots (the binding limit)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "e2e_per_view_dropin": dropin_e2e,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_e2e(sc, vol_h, args, dev):
    """The same pair through trtt_b200_cb3d_batch_ex on pinned host FP64
    arrays, overwriting the outputs (accumulate = 0)."""
    import torch
    from yoricktrtt_b200 import _lib
    lib = _lib.load()
    vol64 = torch.from_numpy(np.ascontiguousarray(vol_h, dtype=np.float64)).pin_memory().numpy()
    det_t = torch.zeros((VIEWS, ND, ND), dtype=torch.float64).pin_memory()
    back_t = torch.zeros((N, N, N), dtype=torch.float64).pin_memory()
    det, back = det_t.numpy(), back_t.numpy()  # same memory, for the C call
    xos = np.ascontiguousarray(sc.xos)
    xsd = np.ascontiguousarray(sc.xsd)

    def call(out, inp, job):
        rc = lib.trtt_b200_cb3d_batch_ex(_lib.dptr(out), _lib.dptr(inp), N, N, N, 1.0, 3, None,
                                         0, 1.0, None, ND, ND, 1.0, 1.0, VIEWS, _lib.dptr(xos),
                                         _lib.dptr(xsd), 4, job, 0)
        _lib.check(rc, "trtt_b200_cb3d_batch_ex")

    def step():
        call(det, vol64, 0)   # det = H vol
        call(back, det, 1)    # back = H^T det

    for _ in range(max(1, min(args.warmup, 2))):
        step()
    steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = (time.perf_counter() - t0) / steps
    nvox, npix = N ** 3, ND * ND * VIEWS
    # per step: the forward copies its input (volume) to the device and its
    # output (detector stack) back; the transpose copies the detector stack
    # in and the volume back (outputs are overwritten, not uploaded)
    h2d = 8 * nvox + 8 * npix
    d2h = 8 * npix + 8 * nvox
    return {"value": 2 * VIEWS / dt, "unit": "projections/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3,
            "path": "trtt_b200_cb3d_batch_ex, accumulate = 0 (host FP64 arrays, reference "
                    "layouts, pinned)"}


def _fan2d_reference():
    """FP64 reference projections for the fan2d workload's parity check."""
    from oracle import oracle
    orc = oracle.get("ref" if oracle.ref_available() else "port")

    def ref(kind, v, img, sc, table, lf):
        img = np.ascontiguousarray(img, dtype=np.float64)
        if kind == "fb2d":
            out = np.zeros(sc.nv)
            orc.p2d("FB2D", out, img, sc, v, 0, table)
            return out
        lf = dict(lf)
        beta = lf.pop("beta")
        out = np.zeros(lf["detectorDimension"])
        orc.lf2d("direct", oracle.LF2DParams(**lf), beta, 0.0, img, out, 1)
        return out

    return ref


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--band-rows", type=int, default=0)
    ap.add_argument("--warps", type=int, default=0)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-parity", action="store_true")
    ap.add_argument("--skip-dense", action="store_true")
    ap.add_argument("--no-symmetry", action="store_true",
                    help="per-view kernels even where views group by turns of the grid")
    ap.add_argument("--workload", default="pair3d",
                    choices=["pair3d", "parallel2d_recon", "fan2d", "cone3d_recon", "gates4d",
                             "learned_warmstart", "learned_eval", "projector_case", "unet_case"],
                    help="pair3d (default) is the benchmark line; the others measure the "
                         "remaining configurations (yoricktrtt_b200/workloads.py)")
    ap.add_argument("--param", action="append", default=[], metavar="KEY=VALUE",
                    help="keyword argument of a --workload function (repeatable)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "pair3d":
        import torch
        from yoricktrtt_b200 import workloads
        torch.cuda.set_device(_env_int("LOCAL_RANK", 0))
        kw = {}
        for kv in args.param:
            k, v = kv.split("=", 1)
            try:
                kw[k] = json.loads(v)
            except ValueError:
                kw[k] = v
        if args.workload == "fan2d":
            kw["reference"] = _fan2d_reference()
        res = getattr(workloads, args.workload)(**kw)
        print(json.dumps({"workload": args.workload, **res}))
        return 0
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
