"""Benchmark: 5.8K ProRes RAW decode + develop frames/s on B200.

Workload (one step = one frame): a 5760x3040 BGGR bitstream-version-0
frame, tile alignment 4, qscale 45, quantization matrix uniform in [4, 63]
(seed 1), default curve, 12-bit mosaic (three cosines + N(0, 24^2) noise,
2 % specular white), 0.5 % of tiles byte-corrupted; decoded with the
Apple-compatible transform and developed to planar Rec.2020 f32. Frames
rotate through a ring of distinct packets; each step writes 210 MB of
planes, more than the 126 MB L2, so no step reads a previous step's data
from L2.

 value  frames/s with the packets resident in HBM, CUDA-event timed on the
        stream the kernels run on, max over ranks.
 e2e    frames/s through the host-buffer C-ABI call prr_decode_develop_host:
        pinned host packet in, pinned host planes out, copies included.
 roofline  the develop kernel's algorithmic bytes (2 B read + 12 B written
        per visible sensel) over its event-timed duration.
 cpu_baseline  the CPU oracle (the crate's algorithm restated in C++,
        threaded like rayon) on a bounded sample of the same frames.

`--impl reference` times the CPU oracle alone (the reference crate is Rust
and cannot be built in this image) on the same workload.
Multi-GPU (torchrun): every rank decodes its own frames (replicas, weak
scaling); no collective is on the data path.
"""

from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 5760, 3040
RING = 3


def make_packets(n: int):
    from proresraw_rs_b200 import synth as S

    rng = np.random.default_rng(1)
    qmat = [int(v) for v in rng.integers(4, 64, 64)]
    pkts = []
    for k in range(n):
        m = S.mosaic(W, H, S.BGGR, seed=100 + k, sigma=24.0, specular=0.02, white=4095)
        spec = S.Spec(W, H, pattern=S.BGGR, alignment=4, quant_matrix=qmat, white_level=4095, version=0,
                      wb=(1.82, 1.41), valid_tiles=True,
                      color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
        pkt = S.encode(spec, m, qscale=45, qscale_seed=k)
        pkt, _ = S.corrupt_tiles(pkt, 0.005, seed=1000 + k)
        pkts.append(pkt)
    return pkts


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profiles():
    """DRAM bytes per develop launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "develop_5760x3040.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
        except OSError:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(pkts, budget_s: float = 15.0):
    """The oracle on the host cores: decode + develop (planar Rec.2020) of the
    bench frames, frames/s over a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    f = O.decode_frame(pkts[0], 0, threads)  # warm-up (page-in, thread start)
    O.develop(f, O.params_new(f.header, f.quantizer), 2, True, threads)
    n, t0 = 0, time.perf_counter()
    while True:
        pkt = pkts[n % len(pkts)]
        f = O.decode_frame(pkt, 0, threads)
        O.develop(f, O.params_new(f.header, f.quantizer), 2, True, threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 200:
            break
    return {"value": n / el, "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": f"{n} frames of the bench workload ({W}x{H}), decode + develop_planar Rec2020, "
                      f"{threads} threads, {el:.1f} s"}


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pkts = make_packets(RING)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    for k in range(args.warmup):
        f = O.decode_frame(pkts[k % RING], 0, threads)
        O.develop(f, O.params_new(f.header, f.quantizer), 2, True, threads)
    t0 = time.perf_counter()
    for k in range(args.steps):
        f = O.decode_frame(pkts[k % RING], 0, threads)
        O.develop(f, O.params_new(f.header, f.quantizer), 2, True, threads)
    el = time.perf_counter() - t0
    v = args.steps / el
    line = {
        "impl": "reference", "metric": "5.8K frames/s decode+develop (bit-exact)", "value": v,
        "unit": "frames/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16+f32", "data": "synthetic",
        "config": {"workload": "5760x3040 BGGR v0 align4 qscale45 qmat[4,63] 0.5% corrupt tiles; "
                               "decode_frame + develop_planar_into(Rec2020)", "frames_in_ring": RING},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} frames, CPU oracle (C++ restatement of the crate's rayon "
                                   f"path; the Rust crate cannot be built here), {threads} threads"},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import _lib

    world, rank, local = dist_setup(args.gpus)
    L = _lib.lib()
    pkts = make_packets(RING)
    infos = [P.frame_info(p) for p in pkts]
    info0 = infos[0]
    n = W * H
    torch.cuda.synchronize()
    # One stream: decode then develop, frame after frame. (Decoding frame k+1
    # on a second stream while frame k develops was measured slower: the
    # latency-bound entropy warps lose issue slots to the develop kernel.)
    s_dec = torch.cuda.Stream()
    s_dev = s_dec
    dev_index = torch.cuda.current_device()
    ctx_dec = C.c_void_p()
    assert L.prr_ctx_create(dev_index, C.c_void_p(s_dec.cuda_stream), C.byref(ctx_dec)) == 0
    ctx_dev = ctx_dec

    # Device-resident packets (padded), scratch, outputs.
    dpk = []
    for p in pkts:
        buf = torch.zeros(L.prr_padded_packet_bytes(len(p)), dtype=torch.uint8, device="cuda")
        buf[: len(p)].copy_(torch.frombuffer(bytearray(p), dtype=torch.uint8))
        dpk.append(buf)
    samples = [torch.empty(info0.coded_width * info0.coded_height, dtype=torch.uint16, device="cuda")
               for _ in range(2)]
    status = torch.zeros(4 * RING, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(info0.ntiles * RING, dtype=torch.int32, device="cuda")
    nscr = L.prr_decode_scratch_bytes(C.byref(info0))
    scratch = torch.empty(nscr, dtype=torch.uint8, device="cuda")
    planes = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    r, g, b = planes[:n], planes[n:2 * n], planes[2 * n:]

    # Parameters per frame come from the host parse (max_qscale is a host
    # walk of the size table, the same value the device scan produces).
    hdrs, params = [], []
    for p in pkts:
        pf = P.parse_frame(p)
        hdrs.append(pf.header)
        params.append(P.DemosaicParams.new(pf.header, P.frame_quantizer(pf))._c())

    dec_done = [torch.cuda.Event() for _ in range(2)]
    dev_done = [torch.cuda.Event() for _ in range(2)]

    def step(k, ev=None):
        i, buf = k % RING, k % 2
        # Decode frame k into code buffer k % 2 once develop k - 2 has read it.
        if k >= 2:
            s_dec.wait_event(dev_done[buf])
        if ev:
            ev[0].record(s_dec)
        rc = L.prr_decode_async(ctx_dec, C.byref(infos[i]), dpk[i].data_ptr(), 0, samples[buf].data_ptr(),
                                status.data_ptr() + 16 * i, skipped.data_ptr() + 4 * info0.ntiles * i,
                                scratch.data_ptr(), nscr)
        assert rc == 0, rc
        if ev:
            ev[1].record(s_dec)
        dec_done[buf].record(s_dec)
        s_dev.wait_event(dec_done[buf])
        if ev:
            ev[2].record(s_dev)
        rc = L.prr_develop(ctx_dev, C.byref(hdrs[i]._c), C.byref(params[i]), 2, samples[buf].data_ptr(), 1,
                           r.data_ptr(), g.data_ptr(), b.data_ptr(), n)
        assert rc == 0, rc
        if ev:
            ev[3].record(s_dev)
        dev_done[buf].record(s_dev)

    for k in range(max(3, args.warmup)):
        step(k)
    torch.cuda.synchronize()
    st = status.cpu().numpy().view(np.uint32).reshape(RING, 4)
    assert np.all(st[:, 0] == 0xFFFFFFFF) and np.all(st[:, 3] == 0)

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = L.prr_kernel_launches()
    with Clocks(torch.cuda.current_device()) as clocks:
        start.record(s_dec)
        for k in range(args.steps):
            step(k, evs[k])
        end.record(s_dev)
        torch.cuda.synchronize()
    launches = L.prr_kernel_launches() - launches0
    if world > 1:
        torch.distributed.barrier()
    ms = start.elapsed_time(end)
    # Per-kernel durations, events on the stream the kernels run on.
    dec_ms = sum(e[0].elapsed_time(e[1]) for e in evs) / args.steps
    dev_ms = sum(e[2].elapsed_time(e[3]) for e in evs) / args.steps
    L.prr_ctx_destroy(ctx_dec)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1000.0)

    e2e_value = None
    if not args.no_e2e:
        e2e_value = measure_e2e(args, L, _lib, pkts, n, world)

    if rank == 0:
        peak, peak_kind = peaks()
        alg_bytes = 2 * n + 12 * n
        achieved = alg_bytes / (dev_ms / 1000.0) / 1e9
        traffic = traffic_from_profiles()
        line = {
            "metric": "5.8K frames/s decode+develop (bit-exact)",
            "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16+f32", "data": "synthetic",
            "config": {"workload": "5760x3040 BGGR v0 align4 qscale45 qmat[4,63] 0.5% corrupt tiles; "
                                   "decode_frame(Apple) + develop_planar_into(Rec2020)",
                       "frames_in_ring": RING, "packet_bytes": [len(p) for p in pkts],
                       "l2": "inputs+outputs > L2 (210 MB planes written per step)",
                       "parallelism": f"replicas x{world}",
                       "decode_ms": dec_ms, "develop_ms": dev_ms},
            "roofline": {"bound": "hbm", "kernel": "k_develop", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": alg_bytes},
            "gpu_launches": int(launches),
        }
        if e2e_value is not None:
            line["e2e"] = {"value": e2e_value, "unit": "frames/s",
                           "h2d_bytes_per_step": int(np.mean([len(p) for p in pkts])),
                           "d2h_bytes_per_step": 12 * n + 16,
                           "note": "prr_decode_develop_host from pinned host memory, 2 host threads, wall clock"}
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(pkts)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def measure_e2e(args, L, _lib, pkts, n, world):
    """Frames/s through prr_decode_develop_host: pinned host packet in,
    pinned host planes out, with two contexts on two host threads so that
    copies overlap kernels. Wall clock, max over ranks."""
    import torch

    host_pkts = []
    for p in pkts:
        hp = torch.empty(len(p), dtype=torch.uint8, pin_memory=True)
        hp.copy_(torch.frombuffer(bytearray(p), dtype=torch.uint8))
        host_pkts.append(hp)
    nthreads = 2
    outs = [torch.empty(3 * n, dtype=torch.float32, pin_memory=True) for _ in range(nthreads)]
    ctxs = []
    for _ in range(nthreads):
        cx = C.c_void_p()
        assert L.prr_ctx_create(torch.cuda.current_device(), None, C.byref(cx)) == 0
        ctxs.append(cx)

    def e2e_worker(tid, frames, errors):
        cx, o = ctxs[tid], outs[tid]
        res, err = _lib.CDecodeResult(), _lib.CError()
        for k in frames:
            hp = host_pkts[k % RING]
            rc = L.prr_decode_develop_host(cx, hp.data_ptr(), hp.numel(), 0, None, 2, 1, o.data_ptr(),
                                           o.data_ptr() + 4 * n, o.data_ptr() + 8 * n, n, C.byref(res),
                                           C.byref(err))
            if rc:
                errors.append(rc)

    def e2e_run(nframes):
        errors = []
        ths = [threading.Thread(target=e2e_worker, args=(i, range(i, nframes, nthreads), errors))
               for i in range(nthreads)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        el = time.perf_counter() - t0
        assert not errors, errors
        return el

    e2e_run(2 * nthreads)
    if world > 1:
        torch.distributed.barrier()
    el = e2e_run(args.steps)
    te = torch.tensor([el], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    e2e_value = world * args.steps / float(te.item())
    for cx in ctxs:
        L.prr_ctx_destroy(cx)
    return e2e_value


# ---------------------------------------------------------------------------
# Mixed-batch workload: 64 frames drawn by seed 2 -- sizes HD / 4K / 5.8K /
# 8K, bitstream version 0 or 1, RGGB or BGGR, qscale in [15, 45], alignment
# in [0, 4]; half full resolution (Apple transform), half reduced (Half,
# Quarter or Eighth; first or averaged greens) -- decoded as one batch by the
# persistent kernel with the bucket's graph, after the autotuner has picked
# the launch shape. One step = one batch.

BATCH_N, BATCH_SEED = 64, 2


def batch_jobs():
    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import synth as S

    items = S.mixed_batch(BATCH_N, seed=BATCH_SEED)
    jobs = [P.BatchJob(it.packet, None if it.scale == 0 else P.Scale(it.scale), P.Idct.APPLE,
                       P.Greens(it.greens)) for it in items]
    return items, jobs


def batch_bytes(items):
    """Algorithmic bytes of a batch: packets read + outputs written."""
    total = 0
    for it in items:
        cw, ch = (it.width + 15) // 16 * 16, (it.height + 15) // 16 * 16
        out = 2 * cw * ch if it.scale == 0 else 6 * (cw >> it.scale) * (ch >> it.scale)
        total += len(it.packet) + out
    return total


def batch_cpu(items, budget_s: float):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    n, t0 = 0, time.perf_counter()
    while True:
        it = items[n % len(items)]
        if it.scale == 0:
            O.decode_frame(it.packet, 0, threads)
        else:
            O.decode_frame_reduced(it.packet, it.scale, it.greens, threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 4 * len(items):
            break
    return n / el, n, el, threads


BATCH_METRIC = "mixed-batch frames/s decode (bit-exact)"
BATCH_WORKLOAD = ("64 frames, seed 2: {1920x1080, 4096x2160, 5760x3040, 8192x4320}, v0/v1, RGGB/BGGR, "
                  "qscale U[15,45], align U[0,4]; half decode_frame(Apple), half decode_frame_reduced "
                  "(Half/Quarter/Eighth, First/Average)")


def run_batch(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import _lib

    world, rank, local = dist_setup(args.gpus)
    L = _lib.lib()
    items, jobs = batch_jobs()
    outs = []
    for it in items:
        cw, ch = (it.width + 15) // 16 * 16, (it.height + 15) // 16 * 16
        n_out = cw * ch if it.scale == 0 else 3 * (cw >> it.scale) * (ch >> it.scale)
        outs.append(torch.empty(n_out, dtype=torch.uint16, device="cuda"))
    dec = P.BatchDecoder()
    res = dec.decode(jobs, outs)
    assert not any(isinstance(r, P.Error) for r in res)
    cfg, tuned_ms = dec.tune(jobs, reps=2)
    for _ in range(max(3, args.warmup)):
        dec.decode(jobs, outs)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = L.prr_kernel_launches()
    dev_ms = []
    with Clocks(torch.cuda.current_device()) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dec.decode(jobs, outs)
            dev_ms.append(dec.last_ms())
        wall = time.perf_counter() - t0
    launches = L.prr_kernel_launches() - launches0
    t = torch.tensor([sum(dev_ms), wall], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max, wall_max = float(t[0].item()), float(t[1].item())
    value = world * args.steps * BATCH_N / (ms_max / 1000.0)
    if rank == 0:
        peak, peak_kind = peaks()
        alg = batch_bytes(items)
        achieved = alg / (ms_max / args.steps / 1000.0) / 1e9
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD, "frames_per_step": BATCH_N,
                       "packet_bytes_per_step": sum(len(it.packet) for it in items),
                       "l2": "inputs+outputs > L2 (about 1 GB written per step)",
                       "parallelism": f"replicas x{world}",
                       "launch_shape": dataclasses.asdict(cfg), "tuned_ms": tuned_ms},
            "roofline": {"bound": "hbm", "kernel": "k_batch_decode", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg},
            "gpu_launches": int(launches),
            "e2e": {"value": world * args.steps * BATCH_N / wall_max, "unit": "frames/s",
                    "h2d_bytes_per_step": sum(len(it.packet) for it in items),
                    "d2h_bytes_per_step": 16 * BATCH_N,
                    "note": "BatchDecoder.decode from host packets: parse, upload, kernels, statuses back; "
                            "frames stay on the device"},
        }
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        if world == 1 and not args.no_cpu_baseline:
            v, n, el, threads = batch_cpu(items, 15.0)
            line["cpu_baseline"] = {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                                    "sample": f"{n} frames of the batch in order, oracle decode, {threads} "
                                              f"threads, {el:.1f} s"}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_batch_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    items, _ = batch_jobs()
    budget = max(10.0, 2.0 * args.steps)
    v, n, el, threads = batch_cpu(items, budget)
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / n * BATCH_N,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "frames_per_step": BATCH_N},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{n} frames of the batch, CPU oracle, {threads} threads, {el:.1f} s"},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="5k8", choices=["5k8", "mixed-batch"],
                    help="5k8: the headline single-frame decode+develop; mixed-batch: 64 uneven frames per step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    args = ap.parse_args()
    if args.workload == "mixed-batch":
        return run_batch_reference(args) if args.impl == "reference" else run_batch(args)
    if args.impl == "reference":
        return run_reference(args)
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
