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
        streams the kernels run on (frame k+1 decodes on a higher-priority
        stream while frame k develops), max over ranks.
 e2e    frames/s through the host-buffer C-ABI call prr_decode_develop_host:
        pinned host packet in, pinned host planes out, copies included.
 roofline  the develop kernel's algorithmic bytes (2 B read + 12 B written
        per visible sensel) over its event-timed duration in the timed
        region, where it shares the SMs with the next frame's decode.
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
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from proresraw_rs_b200 import replicas as R  # noqa: E402

W, H = 5760, 3040
RING = 3
# The workload of the default bench line, in both arms.
WORKLOAD_5K8 = ("5760x3040 BGGR v0 align4 qscale45 qmat[4,63] 0.5% corrupt tiles; "
                "decode_frame(Apple) + develop_planar_into(Rec2020)")
CLIP_WORKLOAD = ("QuickTime clip of {nf} samples ({distinct} distinct 5760x3040 BGGR v0 align4 qscale45 packets, "
                 "0.5% corrupt tiles), file in the page cache; decode_frame (Apple) of every sample")
DNG_WORKLOAD = ("5760x3040 BGGR v0 align4 qscale45 qmat[4,63] 0.5% corrupt tiles; decode_frame (Apple) + "
                "dng::write (code values, LinearizationTable, 256-square LJ92 tiles)")


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


def profile_value(name: str, key: str):
    """A `key: number` line of a committed ncu summary under profiles/, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def traffic_from_profiles(name: str = "develop_5760x3040.md"):
    """DRAM bytes per launch of a kernel from its committed ncu summary
    (a `traffic_bytes_per_launch:` line), if any."""
    return profile_value(name, "traffic_bytes_per_launch")


def nvml_ids(dev: int):
    """The NVML identities of CUDA device `dev`: its UUID and PCI bus id.
    CUDA ordinals and NVML indices differ under a remapped
    CUDA_VISIBLE_DEVICES, so the clock sampler never uses the ordinal."""
    import torch

    p = torch.cuda.get_device_properties(dev)
    uuid = "GPU-" + str(p.uuid)
    pci = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    return uuid, pci


class Clocks:
    """SM clocks and clock-event reasons, read through NVML every 10 ms on a
    thread, with `nvidia-smi -lms 200` beside it; reading only. Samples carry
    their time, so that the summary covers the settle phase (steps run for
    at least a second right before the timed region, so that the clocks
    reach their steady state under this load) and the timed region, and
    counts the samples that fell inside the timed region itself."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, dev: int):
        self.uuid, self.pci = nvml_ids(dev)
        self.proc = None
        # The raw nvidia-smi samples (the line carries their summary).
        out_dir = os.environ.get("PRR_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_{os.getpid()}.csv")
        self.samples = []  # (time, sm_mhz, max_mhz, reasons)
        self._stop = threading.Event()
        self._thread = None
        self.t_timed = None  # perf_counter at the start of the timed region
        self.t_end = None

    def _handle(self, N):
        try:
            return N.nvmlDeviceGetHandleByUUID(self.uuid.encode())
        except Exception:
            return N.nvmlDeviceGetHandleByPciBusId(self.pci.encode())

    def _nvml_loop(self):
        try:
            import pynvml as N

            N.nvmlInit()
            h = self._handle(N)
            bits = [N.nvmlClocksEventReasonHwSlowdown, N.nvmlClocksEventReasonHwThermalSlowdown,
                    N.nvmlClocksEventReasonSwThermalSlowdown, N.nvmlClocksEventReasonSwPowerCap]
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            while True:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), float(sm), float(mx),
                                     [n for n, b in zip(self.NAMES, bits) if r & b]))
                if self._stop.wait(0.01):
                    break
            N.nvmlShutdown()
        except Exception:
            pass

    def timed(self):
        """Mark the start of the timed region."""
        self.t_timed = time.perf_counter()

    def __enter__(self):
        self._thread = threading.Thread(target=self._nvml_loop, daemon=True)
        self._thread.start()
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.uuid,
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.t_end = time.perf_counter()
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        sm, mx, reasons = [], [], set()
        timed = 0
        for t, s_mhz, m_mhz, rs in self.samples:
            sm.append(s_mhz)
            mx.append(m_mhz)
            reasons.update(rs)
            if self.t_timed is not None and t >= self.t_timed:
                timed += 1
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
        except OSError:
            rows = []
        for r in rows:
            if len(r) > 2 and r[1].replace(".", "").isdigit():
                sm.append(float(r[1]))
            if len(r) > 2 and r[2].replace(".", "").isdigit():
                mx.append(float(r[2]))
            reasons.update(self.NAMES[i] for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active")
        if not sm:
            return None
        out = {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx) if mx else None,
               "reasons": sorted(reasons), "samples": len(sm), "timed_region_nvml_samples": timed,
               "window": "settle phase (>= 1 s of steps under the same load) + timed region", "nvml_device": self.uuid}
        if self.t_timed is not None and self.t_end is not None:
            out["settle_s"] = round(self.t_timed - (self.samples[0][0] if self.samples else self.t_timed), 3)
        return out


def settle(step_fn, min_s: float = 1.0, sync=None):
    """Run steps for at least `min_s` of wall time (clocks reach their
    steady state under the load) right before the timed region; returns
    the number of steps run."""
    k, t0 = 0, time.perf_counter()
    while True:
        step_fn(k)
        k += 1
        if k % 8 == 0 or k < 8:
            if sync:
                sync()
            if time.perf_counter() - t0 >= min_s:
                return k


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
        "config": {"workload": WORKLOAD_5K8, "frames_in_ring": RING},
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
    dev_index = torch.cuda.current_device()
    if args.overlap:
        # Two streams: frame k+1 decodes while frame k develops. The decode
        # stream has the higher priority, so the block scheduler gives it
        # each slot a develop CTA frees; --develop-ctas can cap the develop
        # (measured slower: 3 per SM 1860 frames/s, 2 per SM 1463, against
        # 2072 uncapped).
        s_dec = torch.cuda.Stream(priority=-1)
        s_dev = torch.cuda.Stream(priority=0)
    else:
        # One stream: decode then develop, frame after frame.
        s_dec = torch.cuda.Stream()
        s_dev = s_dec
    ctx_dec = C.c_void_p()
    assert L.prr_ctx_create(dev_index, C.c_void_p(s_dec.cuda_stream), C.byref(ctx_dec)) == 0
    ctx_dev = ctx_dec
    if args.overlap:
        ctx_dev = C.c_void_p()
        assert L.prr_ctx_create(dev_index, C.c_void_p(s_dev.cuda_stream), C.byref(ctx_dev)) == 0
        assert L.prr_develop_set_occupancy(ctx_dev, args.develop_ctas) == 0

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
    with Clocks(torch.cuda.current_device()) as clocks:
        settle(step, 1.0, torch.cuda.synchronize)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        launches0 = L.prr_kernel_launches()
        clocks.timed()
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
    if ctx_dev.value != ctx_dec.value:
        L.prr_ctx_destroy(ctx_dev)
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
            "config": {"workload": WORKLOAD_5K8,
                       "frames_in_ring": RING, "packet_bytes": [len(p) for p in pkts],
                       "l2": "inputs+outputs > L2 (210 MB planes written per step)",
                       "parallelism": f"replicas x{world}",
                       "decode_ms": dec_ms, "develop_ms": dev_ms,
                       "streams": ("decode of frame k+1 on a higher-priority stream beside develop of frame k"
                                   + (f" (at most {args.develop_ctas} develop CTAs per SM)" if args.develop_ctas
                                      else "")) if args.overlap else "one stream"},
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
                           "note": f"prr_decode_develop_host from pinned host memory, {args.e2e_threads} host "
                                   "threads, wall clock"}
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        # The develop kernel is bound by instruction issue, not by HBM: its
        # warp instructions per launch (ncu smsp__inst_executed.sum, from the
        # committed capture) over the same event-timed duration, against
        # the SMs' issue rate at the sampled clock (4 schedulers an SM, one
        # warp instruction a cycle each).
        winst = profile_value("develop_5760x3040.md", "warp_instructions_per_launch")
        mhz = (cl or {}).get("sm_mhz") or (cl or {}).get("sm_max_mhz")
        if winst and mhz:
            sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
            issue_peak = sms * 4 * mhz * 1e6
            issue = winst / (dev_ms / 1000.0)
            line["roofline"]["issue"] = {"warp_instructions_per_launch": winst, "achieved_per_s": issue,
                                         "peak_per_s": issue_peak, "frac": issue / issue_peak,
                                         "peak_source": f"{sms} SMs x 4 schedulers x {mhz} MHz"}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(pkts)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def measure_e2e(args, L, _lib, pkts, n, world):
    """Frames/s through prr_decode_develop_host: pinned host packet in,
    pinned host planes out, with a context on each of --e2e-threads host
    threads so that copies overlap kernels. Wall clock, max over ranks."""
    import torch

    host_pkts = []
    for p in pkts:
        hp = torch.empty(len(p), dtype=torch.uint8, pin_memory=True)
        hp.copy_(torch.frombuffer(bytearray(p), dtype=torch.uint8))
        host_pkts.append(hp)
    nthreads = args.e2e_threads
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


def batch_jobs(n=BATCH_N):
    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import synth as S

    items = S.mixed_batch(n, seed=BATCH_SEED)
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
    items, jobs = batch_jobs(args.batch_frames)
    nb = len(items)
    outs = []
    for it in items:
        cw, ch = (it.width + 15) // 16 * 16, (it.height + 15) // 16 * 16
        n_out = cw * ch if it.scale == 0 else 3 * (cw >> it.scale) * (ch >> it.scale)
        outs.append(torch.empty(n_out, dtype=torch.uint16, device="cuda"))
    dec = P.BatchDecoder()
    res = dec.decode(jobs, outs)
    assert not any(isinstance(r, P.Error) for r in res)
    if args.no_tune:
        cfg, tuned_ms = dec.get_config(dec.bucket(jobs)), None
    else:
        cfg, tuned_ms = dec.tune(jobs, reps=2)
    for _ in range(max(3, args.warmup)):
        dec.decode(jobs, outs)
    dev_ms = []
    with Clocks(torch.cuda.current_device()) as clocks:
        settle(lambda k: dec.decode(jobs, outs), 1.0)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        launches0 = L.prr_kernel_launches()
        clocks.timed()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dec.decode(jobs, outs)
            dev_ms.append(dec.last_ms())
        wall = time.perf_counter() - t0
    launches = L.prr_kernel_launches() - launches0
    # End to end: --batch-decoders decoders, each on a stream of its own,
    # take turns, so that the next batches are parsed, staged and uploaded
    # while batch k's kernels run (BatchDecoder.submit / wait).
    bucket = dec.bucket(jobs)
    nd = max(2, args.batch_decoders)
    pipes = []
    for _ in range(nd):
        with torch.cuda.stream(torch.cuda.Stream()):
            dk = P.BatchDecoder()
        dk.set_config(bucket, cfg)
        pipes.append((dk, [torch.empty_like(o) for o in outs]))

    def pipelined(nsteps):
        for st in range(min(nd - 1, nsteps)):
            pipes[st][0].submit(jobs, pipes[st][1])
        for st in range(nsteps):
            if st + nd - 1 < nsteps:
                dk, ok = pipes[(st + nd - 1) % nd]
                dk.submit(jobs, ok)
            res = pipes[st % nd][0].wait()
            assert not any(isinstance(r, P.Error) for r in res)

    pipelined(max(3, args.warmup))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    pipelined(args.steps)
    wall = time.perf_counter() - t0
    t = torch.tensor([sum(dev_ms), wall], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max, wall_max = float(t[0].item()), float(t[1].item())
    value = world * args.steps * nb / (ms_max / 1000.0)
    if rank == 0:
        peak, peak_kind = peaks()
        alg = batch_bytes(items)
        achieved = alg / (ms_max / args.steps / 1000.0) / 1e9
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD.replace("64 frames", f"{nb} frames"), "frames_per_step": nb,
                       "packet_bytes_per_step": sum(len(it.packet) for it in items),
                       "l2": "inputs+outputs > L2 (about 1 GB written per step)",
                       "parallelism": f"replicas x{world}",
                       "launch_shape": dataclasses.asdict(cfg), "tuned_ms": tuned_ms},
            "roofline": {"bound": "hbm", "kernel": "k_batch_decode", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg},
            "gpu_launches": int(launches),
            "e2e": {"value": world * args.steps * nb / wall_max, "unit": "frames/s",
                    "h2d_bytes_per_step": sum(len(it.packet) for it in items),
                    "d2h_bytes_per_step": 16 * nb,
                    "note": "BatchDecoder.submit / wait from host packets (parse, stage, upload, kernels, "
                            f"statuses back), {nd} decoders on streams of their own taking turns so that the next "
                            "batches' uploads overlap a batch's kernels; frames stay on the device"},
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
    items, _ = batch_jobs(args.batch_frames)
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


# ---------------------------------------------------------------------------
# Clip workload: a QuickTime movie of 5760x3040 frames (the headline frames,
# CLIP_DISTINCT distinct packets repeated to CLIP_N samples, 4 samples to a
# chunk) written to the local temp directory, so it sits in the page cache,
# and decoded by the clip pipeline: reader threads read samples into pinned
# memory while the device decodes the previous batch. One step = one pass
# over the whole clip. value: frames over the summed device time of the
# batch kernels; e2e: frames over the wall time of the pass (reads, uploads,
# kernels, statuses back), the frames left decoded in HBM. The batches of
# the two lanes overlap on the device; each counts the part of its kernel
# interval after the previous batch's kernels ended. The sequential
# loop a crate caller writes (read one sample, decode it) is timed beside it
# through the library's host-buffer decode call.

CLIP_N, CLIP_DISTINCT, CLIP_BATCH, CLIP_THREADS = 96, 4, 16, 16
CLIP_METRIC = "clip decode frames/s (movie file -> decoded 5.8K frames in HBM, bit-exact)"


def clip_file(n_frames):
    import tempfile

    from proresraw_rs_b200 import synth_movie as M

    pkts = make_packets(CLIP_DISTINCT)
    path = os.path.join(tempfile.gettempdir(), f"prr_clip_{os.getpid()}.mov")
    M.write_clip(path, [pkts[i % CLIP_DISTINCT] for i in range(n_frames)], per_chunk=4, make="synthetic")
    return path, pkts


def clip_cpu(track, budget_s: float):
    """The oracle on the host cores: read a sample, decode it (all threads)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    O.decode_frame(track.sample(0), 0, threads)
    n, t0 = 0, time.perf_counter()
    while True:
        O.decode_frame(track.sample(n % len(track.samples)), 0, threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 20 * len(track.samples):
            break
    return n / el, n, el, threads


def run_clip(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import _lib
    from proresraw_rs_b200 import clip as CL
    from proresraw_rs_b200 import mov

    world, rank, local = dist_setup(args.gpus)
    L = _lib.lib()
    path, pkts = clip_file(args.clip_frames)
    try:
        track = mov.read_video_track(path)
        nf = len(track.samples)
        dec = CL.ClipDecoder(track, args.clip_batch, args.clip_threads)

        def passes(n, check=False):
            # n passes over the clip back to back: each pass queues the next
            # at its first batch, so that the next pass's first reads and
            # uploads overlap this pass's last batches.
            frames, dev_ms = 0, 0.0
            it = dec.batches()
            for p in range(n):
                for k, batch in enumerate(it):
                    if k == 0 and p + 1 < n:
                        dec.queue()
                    if check:
                        assert not any(isinstance(f, Exception) for f in batch.frames)
                    frames += len(batch.frames)
                    dev_ms += batch.busy_ms
                if p + 1 < n:
                    it = dec.queued_batches()
            return frames, dev_ms

        assert passes(2, check=True)[0] == 2 * nf
        passes(max(3, args.warmup))
        with Clocks(torch.cuda.current_device()) as clocks:
            settle(lambda k: passes(1), 1.0, torch.cuda.synchronize)
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            launches0 = L.prr_kernel_launches()
            clocks.timed()
            t0 = time.perf_counter()
            dev_total = passes(args.steps)[1]
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        launches = L.prr_kernel_launches() - launches0
        t = torch.tensor([dev_total, wall], dtype=torch.float64, device="cuda")
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_max, wall_max = float(t[0].item()), float(t[1].item())
        # The sequential loop: read one sample, decode it from the host buffer.
        seq_n = min(nf, 48)
        ctx = P.context()
        info = P.frame_info(pkts[0])
        out = torch.empty(info.coded_width * info.coded_height, dtype=torch.uint16, device="cuda")
        res, err = _lib.CDecodeResult(), _lib.CError()
        buf = bytearray(max(s.size for s in track.samples))
        cbuf = (C.c_uint8 * len(buf)).from_buffer(buf)
        for _ in range(2):
            track.read_at(track.samples[0].offset, memoryview(buf)[:track.samples[0].size])
            L.prr_decode(ctx, C.addressof(cbuf), track.samples[0].size, 0, out.data_ptr(), out.numel(),
                         C.byref(res), C.byref(err))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for i in range(seq_n):
            s = track.samples[i]
            track.read_at(s.offset, memoryview(buf)[:s.size])
            rc = L.prr_decode(ctx, C.addressof(cbuf), s.size, 0, out.data_ptr(), out.numel(), C.byref(res),
                              C.byref(err))
            assert rc == 0
        seq_fps = seq_n / (time.perf_counter() - t1)
        if rank == 0:
            peak, peak_kind = peaks()
            cw, ch = info.coded_width, info.coded_height
            alg = sum(s.size for s in track.samples) + 2 * cw * ch * nf
            achieved = alg / (ms_max / args.steps / 1000.0) / 1e9
            h2d = sum(s.size for s in track.samples)
            line = {
                "metric": CLIP_METRIC, "value": world * args.steps * nf / (ms_max / 1000.0), "unit": "frames/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u16", "data": "synthetic",
                "config": {"workload": CLIP_WORKLOAD.format(nf=nf, distinct=CLIP_DISTINCT),
                           "frames_per_step": nf, "frames_per_batch": args.clip_batch,
                           "reader_threads": args.clip_threads, "clip_bytes": os.path.getsize(path),
                           "l2": f"{2 * cw * ch * nf / 1e9:.1f} GB of code values written per pass, more than L2",
                           "parallelism": f"replicas x{world}",
                           "sequential_read_then_decode_fps": seq_fps},
                "roofline": {"bound": "hbm", "kernel": "k_batch_decode", "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                             "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg},
                "gpu_launches": int(launches),
                "e2e": {"value": world * args.steps * nf / wall_max, "unit": "frames/s",
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 16 * nf,
                        "note": "ClipDecoder.batches over the movie file: positional reads into pinned memory, "
                                "uploads, kernels, statuses back; each pass queues the next (prr_clip_queue); "
                                "frames stay on the device"},
            }
            cl = clocks.summary()
            if cl:
                line["clocks"] = cl
            if world == 1 and not args.no_cpu_baseline:
                v, n, el, threads = clip_cpu(track, 12.0)
                line["cpu_baseline"] = {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                                        "sample": f"{n} samples read from the clip and decoded by the oracle, "
                                                  f"{threads} threads, {el:.1f} s"}
            print(json.dumps(line), flush=True)
        dec.close()
        track.close()
    finally:
        os.remove(path)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_clip_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from proresraw_rs_b200 import mov

    path, _ = clip_file(args.clip_frames)
    try:
        with mov.read_video_track(path) as track:
            v, n, el, threads = clip_cpu(track, max(10.0, 0.5 * args.steps))
    finally:
        os.remove(path)
    line = {
        "impl": "reference", "metric": CLIP_METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / n * args.clip_frames,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": CLIP_WORKLOAD.format(nf=args.clip_frames, distinct=CLIP_DISTINCT),
                   "frames_per_step": args.clip_frames},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{n} samples read and decoded by the CPU oracle, {threads} threads, {el:.1f} s"},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# DNG workload: the headline 5760x3040 frames exported as the crate's DNG
# files (code values + LinearizationTable, 256-square lossless JPEG tiles).
# One step = one frame. value: frames over the device time of the decode and
# the tile encoder with packets resident in HBM (frame k+1 decodes on a
# higher-priority stream while frame k's tiles are encoded); e2e: frames over the wall
# time of prr_decode (host packet) + prr_dng_write (tiles encoded on the
# device, brought back, the TIFF container written on the host), the file's
# bytes in host memory, on several host threads.

DNG_METRIC = "5.8K frames/s decode + DNG export (lossless JPEG tiles, bit-exact)"


def dng_cpu(pkts, budget_s: float):
    """The oracle on the host cores: decode, cut and encode every tile."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    f = O.decode_frame(pkts[0], 0, threads)
    n, t0 = 0, time.perf_counter()
    while True:
        f = O.decode_frame(pkts[n % len(pkts)], 0, threads)
        O.lj92_tiles(f.samples, W, H, stride=f.header.coded_width, threads=threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 200:
            break
    return n / el, n, el, threads


def run_dng(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import _lib

    world, rank, local = dist_setup(args.gpus)
    L = _lib.lib()
    pkts = make_packets(RING)
    infos = [P.frame_info(p) for p in pkts]
    info0 = infos[0]
    # Frame k+1 decodes on a higher-priority stream while frame k's tiles
    # are encoded (two code-value buffers), as in the headline workload.
    dev_index = torch.cuda.current_device()
    s_dec = torch.cuda.Stream(priority=-1) if args.overlap else torch.cuda.Stream()
    s = torch.cuda.Stream(priority=0) if args.overlap else s_dec
    ctx_dec, ctx = C.c_void_p(), C.c_void_p()
    assert L.prr_ctx_create(dev_index, C.c_void_p(s_dec.cuda_stream), C.byref(ctx_dec)) == 0
    assert L.prr_ctx_create(dev_index, C.c_void_p(s.cuda_stream), C.byref(ctx)) == 0
    dpk = []
    for p in pkts:
        buf = torch.zeros(L.prr_padded_packet_bytes(len(p)), dtype=torch.uint8, device="cuda")
        buf[: len(p)].copy_(torch.frombuffer(bytearray(p), dtype=torch.uint8))
        dpk.append(buf)
    sbufs = [torch.empty(info0.coded_width * info0.coded_height, dtype=torch.uint16, device="cuda")
             for _ in range(2)]
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(info0.ntiles, dtype=torch.int32, device="cuda")
    nscr = L.prr_decode_scratch_bytes(C.byref(info0))
    scratch = torch.empty(nscr, dtype=torch.uint8, device="cuda")
    ntiles = -(-W // 256) * -(-H // 256)
    cap = ntiles * L.prr_lj92_tile_bound(256)
    tiles = torch.empty(cap, dtype=torch.uint8, device="cuda")
    offsets = torch.zeros(ntiles + 1, dtype=torch.int64, device="cuda")
    stride = info0.coded_width
    dec_done = [torch.cuda.Event() for _ in range(2)]
    enc_done = [torch.cuda.Event() for _ in range(2)]

    def step(k, ev=None):
        i, b = k % RING, k % 2
        if k >= 2:
            s_dec.wait_event(enc_done[b])  # the buffer's previous frame is encoded
        if ev:
            ev[0].record(s_dec)
        assert L.prr_decode_async(ctx_dec, C.byref(infos[i]), dpk[i].data_ptr(), 0, sbufs[b].data_ptr(),
                                  status.data_ptr(), skipped.data_ptr(), scratch.data_ptr(), nscr) == 0
        if ev:
            ev[1].record(s_dec)
        dec_done[b].record(s_dec)
        s.wait_event(dec_done[b])
        if ev:
            ev[3].record(s)
        assert L.prr_lj92_encode(ctx, sbufs[b].data_ptr(), W, H, stride, 256, tiles.data_ptr(), cap,
                                 offsets.data_ptr()) == 0
        if ev:
            ev[2].record(s)
        enc_done[b].record(s)

    for k in range(max(3, args.warmup)):
        step(k)
    torch.cuda.synchronize()
    tile_bytes = int(offsets[-1].item())
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clocks:
        settle(step, 1.0, torch.cuda.synchronize)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        launches0 = L.prr_kernel_launches()
        clocks.timed()
        start.record(s_dec)
        for k in range(args.steps):
            step(k, evs[k])
        end.record(s)
        torch.cuda.synchronize()
    launches = L.prr_kernel_launches() - launches0
    ms = start.elapsed_time(end)
    dec_ms = sum(e[0].elapsed_time(e[1]) for e in evs) / args.steps
    lj_ms = sum(e[3].elapsed_time(e[2]) for e in evs) / args.steps
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())

    # End to end: host packet -> DNG bytes in host memory, on DNG_THREADS
    # host threads with a context each (one thread's container writing
    # overlaps another's kernels).
    clip = _lib.CDngClip()
    clip.make, clip.fps_num, clip.fps_den, clip.orientation = b"synthetic", 30, 1, 1
    hbufs = []
    for p in pkts:
        hp = torch.empty(len(p), dtype=torch.uint8, pin_memory=True)
        hp.copy_(torch.frombuffer(bytearray(p), dtype=torch.uint8))
        hbufs.append(hp)
    nthreads = args.dng_threads
    ectx, esamples, efiles = [], [], []
    for _ in range(nthreads):
        cx = C.c_void_p()
        assert L.prr_ctx_create(torch.cuda.current_device(), None, C.byref(cx)) == 0
        ectx.append(cx)
        esamples.append(torch.empty(info0.coded_width * info0.coded_height, dtype=torch.uint16, device="cuda"))
        # A reused pinned file buffer per thread, as a writer that saves the
        # files would keep (twice the raw size: LJ92 never doubles it here).
        efiles.append(torch.empty(4 * W * H, dtype=torch.uint8, pin_memory=True))
    file_bytes = []

    def e2e_worker(tid, frames, errors):
        cx, smp, fb = ectx[tid], esamples[tid], efiles[tid]
        res, err = _lib.CDecodeResult(), _lib.CError()
        for k in frames:
            hp = hbufs[k % RING]
            rc = L.prr_decode(cx, hp.data_ptr(), hp.numel(), 0, smp.data_ptr(), smp.numel(), C.byref(res),
                              C.byref(err))
            nb = C.c_size_t()
            if rc == 0:
                rc = L.prr_dng_write_into(cx, C.byref(res.header), smp.data_ptr(), 0, 1, C.byref(clip),
                                          fb.data_ptr(), fb.numel(), C.byref(nb))
            if rc:
                errors.append(rc)
                continue
            file_bytes.append(nb.value)

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
    e2e_n = max(args.steps, 4 * nthreads)
    e2e_wall = e2e_run(e2e_n)
    te = torch.tensor([e2e_wall], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    e2e_wall = float(te.item())
    for cx in ectx:
        L.prr_ctx_destroy(cx)
    L.prr_ctx_destroy(ctx_dec)
    L.prr_ctx_destroy(ctx)
    if rank == 0:
        peak, peak_kind = peaks()
        # The tile encoder's algorithmic bytes: the visible samples read,
        # the streams written.
        alg = 2 * W * H + tile_bytes
        achieved = alg / (lj_ms / 1000.0) / 1e9
        line = {
            "metric": DNG_METRIC, "value": world * args.steps / (ms_max / 1000.0), "unit": "frames/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
            "data": "synthetic",
            "config": {"workload": DNG_WORKLOAD,
                       "frames_in_ring": RING, "tiles_per_frame": ntiles, "tile_bytes_per_frame": tile_bytes,
                       "dng_file_bytes": file_bytes[-1] if file_bytes else None,
                       "l2": "35 MB of code values and about 20 MB of streams a frame; 3 distinct frames (not "
                             "larger than L2 together: a frame's decode output is re-read by the encoder)",
                       "parallelism": f"replicas x{world}", "decode_ms": dec_ms, "lj92_ms": lj_ms,
                       "streams": "decode of frame k+1 on a higher-priority stream beside frame k's tiles"
                                  if args.overlap else "one stream"},
            "roofline": {"bound": "hbm", "kernel": "k_lj92_encode<256>", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_from_profiles("lj92_tiles_5760x3040.md"),
                         "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg},
            "gpu_launches": int(launches),
            "e2e": {"value": world * e2e_n / e2e_wall, "unit": "frames/s",
                    "h2d_bytes_per_step": int(np.mean([len(p) for p in pkts])),
                    "d2h_bytes_per_step": tile_bytes + 8 * (ntiles + 1) + 16,
                    "note": f"prr_decode from a pinned host packet + prr_dng_write_into a reused pinned file "
                            f"buffer: the DNG file's bytes in host memory, {nthreads} host threads with a context "
                            f"each, wall clock"},
        }
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        if world == 1 and not args.no_cpu_baseline:
            v, n, el, threads = dng_cpu(pkts, 15.0)
            line["cpu_baseline"] = {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                                    "sample": f"{n} frames: oracle decode + oracle LJ92 tiles (the crate's encoder "
                                              f"restated), {threads} threads, {el:.1f} s; the TIFF container not "
                                              "included"}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_dng_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    pkts = make_packets(RING)
    v, n, el, threads = dng_cpu(pkts, max(10.0, 0.2 * args.steps))
    line = {
        "impl": "reference", "metric": DNG_METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": DNG_WORKLOAD},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{n} frames, CPU oracle decode + LJ92 tiles, {threads} threads, {el:.1f} s"},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Learned develop workloads. The surrogate is trained here, on the device,
# by the library's own kernels: 4000 random 512x512 crops of synthetic
# 4096x2160 RGGB frames (the mosaic generator with noise sigma uniform in
# [4, 32], qscale uniform in [15, 45]) developed by the plain GPU path, Adam
# at lr 1e-3, batch 32. One step of the "learned" workload = one held-out
# 4096x2160 frame developed to planar Rec.2020 by the network (device-
# resident codes); the plain develop of the same frames is timed beside it.

LEARN_W, LEARN_H = 4096, 2160
LEARN_TRAIN_FRAMES, LEARN_HELD = 12, 16


def learn_frame(seed, rng):
    from proresraw_rs_b200 import synth as S

    sigma, q = float(rng.uniform(4, 32)), int(rng.integers(15, 46))
    m = S.mosaic(LEARN_W, LEARN_H, S.RGGB, seed=seed, sigma=sigma, white=4095)
    spec = S.Spec(LEARN_W, LEARN_H, pattern=S.RGGB, alignment=2, white_level=4095, version=1, valid_tiles=True,
                  wb=(1.9, 1.4), color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
    return S.encode(spec, m, qscale=q, qscale_seed=seed), sigma, q


def sg_flops_per_frame(w, h):
    """Algorithmic FLOPs of the network per frame: 5 input channels, six
    32-channel 3x3 layers, a 12-channel head, per half-resolution pixel."""
    return 2 * 9 * (5 * 32 + 5 * 32 * 32 + 32 * 12) * ((w + 1) // 2) * ((h + 1) // 2)


def sg_flops_executed_per_frame(w, h):
    """FLOPs the tensor cores execute per frame: the kernels' input layer
    takes 16 channels (the network's inputs plus engineered and zero
    channels) and the head is 16 wide (12 used)."""
    return 2 * 9 * (16 * 32 + 5 * 32 * 32 + 32 * 16) * ((w + 1) // 2) * ((h + 1) // 2)


def tensor_peak(sustained=False):
    key = "bf16_tflops_sustained" if sustained else "bf16_tflops"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)[key]), f"measured {key}"
    except Exception:
        return (1400.0 if sustained else 1590.0), "fallback"


def train_for_bench(P, L, epochs, log=None):
    rng = np.random.default_rng(0)
    frames = [P.decode_frame(learn_frame(1000 + k, rng)[0]) for k in range(LEARN_TRAIN_FRAMES)]
    t0 = time.perf_counter()
    s, hist = L.train_surrogate(frames, crops=4000, batch=32, crop=512, epochs=epochs, lr=1e-3, seed=0, log=log)
    import torch

    torch.cuda.synchronize()
    return s, hist, time.perf_counter() - t0


def run_learned(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import learned as L

    world, rank, local = dist_setup(args.gpus)
    s, hist, train_s = train_for_bench(P, L, args.epochs)
    rng = np.random.default_rng(4242)
    held = [learn_frame(2000 + k, rng) for k in range(LEARN_HELD)]
    frames = [P.decode_frame(pk) for pk, _, _ in held]
    n = LEARN_W * LEARN_H
    out = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    dp = s.device()
    prms = [P.DemosaicParams.new(f.header, f.quantizer()) for f in frames]
    psnrs, maxabs, fb = [], [], 0
    for f, prm in zip(frames, prms):
        fb += L.develop_learned_planar_into(f, prm, P.Stage.REC2020, s, out, dev_params=dp)
        got = np.stack([o.cpu().numpy() for o in out])
        plain = P.develop_planar(f, prm, P.Stage.REC2020)
        want = np.stack([p.cpu().numpy() for p in plain.planes])
        psnrs.append(L.psnr(got, want))
        maxabs.append(L.max_abs(got, want))
    tiles = ((LEARN_W + 31) // 32) * ((LEARN_H + 31) // 32) * len(frames)
    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        for k in range(max(3, args.warmup)):
            fn(k)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(steps):
            fn(k)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def learned_step(k):
        f = frames[k % len(frames)]
        L.develop_learned_planar_into(f, prms[k % len(frames)], P.Stage.REC2020, s, out, dev_params=dp,
                                      count_fallback=False)

    def plain_step(k):
        f = frames[k % len(frames)]
        P.develop_planar_into(f, prms[k % len(frames)], P.Stage.REC2020, out)

    with Clocks(torch.cuda.current_device()) as clocks:
        settle(learned_step, 1.0, torch.cuda.synchronize)
        torch.cuda.synchronize()
        launches0 = P.kernel_launches()
        clocks.timed()
        ms_learned = timed(learned_step, args.steps)
    launches = P.kernel_launches() - launches0
    ms_plain = timed(plain_step, args.steps)
    ms_l, ms_p = R.reduce_max(ms_learned), R.reduce_max(ms_plain)
    # End to end: host packet in, decode, learned develop, planes to pinned
    # host memory; --e2e-threads host threads, each on a stream (and so a
    # context) of its own, so that one frame's copies overlap another's
    # kernels.
    nthreads = args.e2e_threads
    streams = [torch.cuda.Stream() for _ in range(nthreads)]
    hosts = [torch.empty(3 * n, dtype=torch.float32, pin_memory=True) for _ in range(nthreads)]
    outs_t = [[torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)] for _ in range(nthreads)]

    def e2e_worker(tid, ks, errors):
        try:
            with torch.cuda.stream(streams[tid]):
                for k in ks:
                    f = P.decode_frame(held[k % len(held)][0])
                    L.develop_learned_planar_into(f, prms[k % len(frames)], P.Stage.REC2020, s, outs_t[tid],
                                                  dev_params=dp)
                    for c in range(3):
                        hosts[tid][c * n:(c + 1) * n].copy_(outs_t[tid][c], non_blocking=True)
                    streams[tid].synchronize()
        except Exception as e:  # noqa: BLE001 -- reported after the join
            errors.append(e)

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
    e2e_n = max(4 * nthreads, args.steps)
    e2e_s = R.reduce_max(e2e_run(e2e_n))
    if rank == 0:
        peak, pk = tensor_peak()
        speak, spk = tensor_peak(sustained=True)
        flops = sg_flops_per_frame(LEARN_W, LEARN_H)
        xflops = sg_flops_executed_per_frame(LEARN_W, LEARN_H)
        line = {
            "metric": "learned develop frames/s (4096x2160 to planar Rec.2020)", "value": world * 1000.0 / ms_l,
            "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_l,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (f32 accumulate)",
            "data": "synthetic",
            "config": {"workload": "surrogate develop of 16 held-out 4096x2160 RGGB frames (sigma U[4,32], qscale "
                                   "U[15,45]); trained on 4000 512x512 crops, batch 32, Adam lr 1e-3",
                       "train_epochs": args.epochs, "train_seconds": train_s,
                       "train_loss_first_last": [hist[0], hist[-1]],
                       "plain_develop_ms": ms_p, "plain_develop_frames_per_s": 1000.0 / ms_p,
                       "learned_over_plain_speed": ms_p / ms_l,
                       "psnr_db_vs_plain": {"min": min(psnrs), "mean": float(np.mean(psnrs)), "max": max(psnrs)},
                       "max_abs_vs_plain": max(maxabs),
                       "fallback_tiles": fb, "fallback_rate": fb / tiles,
                       "l2": "outputs (106 MB planes) and activations (141 MB in and out of each fused pair of "
                             "layers) exceed L2",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "tensor",
                         "kernel": "learned develop (three fused pairs of conv layers, the head, packing)",
                         "achieved": flops / (ms_l / 1000.0) / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": flops / (ms_l / 1000.0) / 1e12 / peak, "traffic": None, "peak_source": pk,
                         "flops_counted": "algorithmic: the network as specified (5 input channels, 12-wide head)",
                         "algorithmic_flops_per_frame": flops,
                         "executed_flops_per_frame": xflops,
                         "executed": {"achieved": xflops / (ms_l / 1000.0) / 1e12,
                                      "frac": xflops / (ms_l / 1000.0) / 1e12 / peak,
                                      "frac_of_sustained": xflops / (ms_l / 1000.0) / 1e12 / speak,
                                      "sustained_peak": speak, "sustained_peak_source": spk}},
            "gpu_launches": int(launches),
            "e2e": {"value": world * e2e_n / e2e_s, "unit": "frames/s",
                    "h2d_bytes_per_step": int(np.mean([len(h[0]) for h in held])), "d2h_bytes_per_step": 12 * n,
                    "note": f"decode_frame from a host packet, learned develop, planes copied to pinned host "
                            f"memory; {nthreads} host threads with a stream each, wall clock"},
        }
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        if world == 1 and not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            import _oracle as O

            threads = os.cpu_count() or 1
            nf, t0 = 0, time.perf_counter()
            while time.perf_counter() - t0 < 10.0 and nf < 16:
                of = O.decode_frame(held[nf][0], 0, threads)
                O.develop(of, O.params_new(of.header, of.quantizer), 2, True, threads)
                nf += 1
            el = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": nf / el, "unit": "frames/s", "cores": threads, "kind": "port",
                                    "sample": f"{nf} held-out frames, oracle decode + plain develop (the reference "
                                              f"has no learned develop), {threads} threads, {el:.1f} s"}
        if args.save_model:
            s.save(args.save_model)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


# 8K stream: 16 frames of 8192x4320 RGGB, version 1, qscale uniform in
# [15, 45] (seed 4), noise sigma uniform in [4, 32]. One step = the 16
# frames: one batch decode (the batch kernel's graph, replayed), then per
# frame linearize and the learned develop to planar Rec.2020 into
# preallocated device buffers, captured once as a CUDA graph and replayed.

STREAM_W, STREAM_H, STREAM_N = 8192, 4320, 16


def run_stream(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import learned as L
    from proresraw_rs_b200 import synth as S

    world, rank, local = dist_setup(args.gpus)
    if args.model and os.path.exists(args.model):
        s = L.Surrogate.load(args.model)
        train_s = 0.0
    else:
        s, _, train_s = train_for_bench(P, L, args.epochs)
    rng = np.random.default_rng(4)
    pkts = []
    for k in range(STREAM_N):
        sigma, q = float(rng.uniform(4, 32)), int(rng.integers(15, 46))
        m = S.mosaic(STREAM_W, STREAM_H, S.RGGB, seed=4000 + k, sigma=sigma, white=4095)
        spec = S.Spec(STREAM_W, STREAM_H, pattern=S.RGGB, version=1, white_level=4095, valid_tiles=True,
                      wb=(1.9, 1.4), color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
        pkts.append(S.encode(spec, m, qscale=q, qscale_seed=k))
    pkts = R.shard(pkts, rank, world) if world > 1 else pkts
    nfr = len(pkts)
    cw, ch = STREAM_W, STREAM_H
    n = STREAM_W * STREAM_H
    # Two sets of code buffers, each with its decoder (on a stream of its
    # own) and its captured develop graph: step k+1's batch decode runs
    # beside step k's develop.
    codes = [[torch.empty(cw * ch, dtype=torch.uint16, device="cuda") for _ in range(nfr)] for _ in range(2)]
    lin = torch.empty(n, dtype=torch.uint16, device="cuda")
    planes = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    dstreams, decs = [torch.cuda.Stream() for _ in range(2)], []
    for st_ in dstreams:
        with torch.cuda.stream(st_):
            decs.append(P.BatchDecoder())
    jobs = [P.BatchJob(p) for p in pkts]
    frames = []
    for k in range(2):
        res = decs[k].decode(jobs, codes[k])
        assert not any(isinstance(r, P.Error) for r in res)
        frames.append(res)
    prms = [P.DemosaicParams.new(f.header, f.quantizer()) for f in frames[0]]
    dp = s.device()
    sur = L.Surrogate(s.params, s.noise_lo, s.noise_hi)
    side = torch.cuda.Stream()

    def develop_all(fr, learned=True):
        for f, prm in zip(fr, prms):
            f.linearize_into(lin)
            if learned:
                L.develop_learned_planar_into(f, prm, P.Stage.REC2020, sur, planes, dev_params=dp,
                                              count_fallback=False)
            else:
                P.develop_planar_into(f, prm, P.Stage.REC2020, planes)

    # Warm up (allocations happen here), then capture the develop stage.
    with torch.cuda.stream(side):
        develop_all(frames[0])
        develop_all(frames[0], False)
    torch.cuda.synchronize()
    graphs = []
    for k in range(2):
        g = torch.cuda.CUDAGraph()
        k0 = P.kernel_launches()
        with torch.cuda.graph(g, stream=side):
            develop_all(frames[k])
        kernels_per_replay = P.kernel_launches() - k0  # launches recorded while capturing
        graphs.append(g)
    gp = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gp, stream=side):
        develop_all(frames[0], False)
    torch.cuda.synchronize()
    developed = [torch.cuda.Event(), torch.cuda.Event()]

    def run_steps(nsteps):
        dec_ms = 0.0
        decs[0].submit(jobs, codes[0])
        for st in range(nsteps):
            cur, nxt = st % 2, 1 - st % 2
            res = decs[cur].wait()
            assert not any(isinstance(r, P.Error) for r in res)
            dec_ms += decs[cur].last_ms()
            if st + 1 < nsteps:
                if st >= 1:
                    dstreams[nxt].wait_event(developed[nxt])  # step k-1's develop has read these codes
                decs[nxt].submit(jobs, codes[nxt])
            with torch.cuda.stream(side):
                graphs[cur].replay()
                developed[cur].record(side)
        side.synchronize()
        return dec_ms

    run_steps(max(3, args.warmup))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clocks:
        settle(lambda k: run_steps(1), 1.0, torch.cuda.synchronize)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        launches0 = P.kernel_launches()
        clocks.timed()
        t0 = time.perf_counter()
        e0.record(side)
        dec_ms = run_steps(args.steps)
        e1.record(side)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    span_ms = e0.elapsed_time(e1)
    launches = P.kernel_launches() - launches0 + kernels_per_replay * args.steps
    # The develop stage alone, and the plain develop in the same pipeline,
    # for comparison.

    def replay_ms(graph, reps):
        t = 0.0
        for _ in range(reps):
            e0.record(side)
            with torch.cuda.stream(side):
                graph.replay()
            e1.record(side)
            torch.cuda.synchronize()
            t += e0.elapsed_time(e1)
        return t / reps

    dev_ms = replay_ms(graphs[0], max(2, args.steps // 2))
    pd = replay_ms(gp, max(2, args.steps // 2))
    ms_step = R.reduce_max(span_ms / args.steps)
    wall_step = R.reduce_max(wall / args.steps)
    nall = int(R.reduce_sum(nfr))
    if rank == 0:
        peak, pk = peaks()
        # Bytes per frame of the pipeline: packet + codes written, codes read
        # twice (linearize, develop pack), linear values written, planes written.
        pkt_bytes = float(np.mean([len(p) for p in pkts]))
        alg = pkt_bytes + 2 * cw * ch + 2 * 2 * cw * ch + 2 * n + 12 * n
        line = {
            "metric": "8K stream frames/s (decode + linearize + learned develop to planar Rec.2020)",
            "value": nall / (ms_step / 1000.0), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16 decode, bf16 network (f32 accumulate)", "data": "synthetic",
            "config": {"workload": "16 x 8192x4320 RGGB v1, qscale U[15,45] seed 4, sigma U[4,32]; batch decode "
                                   "graph + per-frame linearize + learned develop graph",
                       "frames_per_step": nfr, "decode_ms_per_step": dec_ms / args.steps,
                       "develop_ms_per_step": dev_ms, "plain_develop_pipeline_ms_per_step": pd,
                       "streams": "step k+1's batch decode (a second decoder and code buffers) beside step k's "
                                  "develop graph; value over the device span of the timed steps",
                       "model_trained_seconds": train_s, "parallelism": f"replicas x{world}",
                       "l2": "every frame's planes (425 MB) exceed L2"},
            "roofline": {"bound": "hbm", "kernel": "whole pipeline", "achieved": alg * nfr / (ms_step / 1000.0) / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg * nfr / (ms_step / 1000.0) / 1e9 / peak,
                         "traffic": None, "peak_source": f"{pk} hbm_gbs", "algorithmic_bytes_per_frame": alg},
            "gpu_launches": int(launches),
            "e2e": {"value": nall / wall_step, "unit": "frames/s", "h2d_bytes_per_step": int(sum(len(p) for p in pkts)),
                    "d2h_bytes_per_step": 16 * nfr,
                    "note": "batch decode from host packets (parse, upload, graph) + develop graph, pipelined "
                            "over two decoders; planes stay on the device"},
        }
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        print(json.dumps(line), flush=True)
    del graphs, gp
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Linearize workload: Frame::linearize_into of decoded 5760x3040 frames
# (code values through the frame's 8-point curve, src/curve.rs:14-33,
# src/decoder.rs:197-216), device-resident; a ring of LIN_RING frames of
# code values and outputs (4 x 70 MB, more than L2). One step = one frame.
LIN_RING = 4
LIN_WORKLOAD = ("5760x3040 BGGR v0 align4 qscale45 frames (decoded code values, curve of the header); "
                "Frame::linearize_into")


def run_linearize(args):
    import torch

    import proresraw_rs_b200 as P
    from proresraw_rs_b200 import _lib

    world, rank, local = dist_setup(args.gpus)
    L = _lib.lib()
    pkts = make_packets(RING)
    frames = [P.decode_frame(pkts[k % RING]) for k in range(LIN_RING)]
    n = W * H
    outs = [torch.empty(n, dtype=torch.uint16, device="cuda") for _ in range(LIN_RING)]
    s = torch.cuda.Stream()
    ctx = C.c_void_p()
    assert L.prr_ctx_create(torch.cuda.current_device(), C.c_void_p(s.cuda_stream), C.byref(ctx)) == 0
    torch.cuda.synchronize()

    def step(k, ev=None):
        f, o = frames[k % LIN_RING], outs[k % LIN_RING]
        if ev:
            ev[0].record(s)
        assert L.prr_linearize(ctx, C.byref(f.header._c), f.samples.data_ptr(), o.data_ptr(), n) == 0
        if ev:
            ev[1].record(s)

    for k in range(max(3, args.warmup)):
        step(k)
    torch.cuda.synchronize()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    want = O.decode_frame(pkts[0], 0, os.cpu_count() or 1).linearize(os.cpu_count() or 1)
    assert np.array_equal(outs[0].cpu().numpy().view(np.uint16), want.reshape(-1)), "linearize differs"
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clocks:
        settle(step, 1.0, torch.cuda.synchronize)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        launches0 = L.prr_kernel_launches()
        clocks.timed()
        start.record(s)
        for k in range(args.steps):
            step(k)
        end.record(s)
        torch.cuda.synchronize()
    launches = L.prr_kernel_launches() - launches0
    ms = R.reduce_max(start.elapsed_time(end))
    # One kernel a step, back to back on one stream: the kernel's average
    # duration is the timed region over the steps (events around each
    # launch would add their own gaps to a 20 µs kernel).
    lin_ms = ms / args.steps
    value = world * args.steps / (ms / 1000.0)
    # End to end: host code values in (pinned), linear values out (pinned).
    e2e = None
    if not args.no_e2e:
        hin = torch.empty(n, dtype=torch.uint16, pin_memory=True)
        hin.copy_(frames[0].samples.cpu())
        hout = torch.empty(n, dtype=torch.uint16, pin_memory=True)
        din, dout = torch.empty(n, dtype=torch.uint16, device="cuda"), outs[0]
        hdr = frames[0].header._c

        def e2e_step():
            with torch.cuda.stream(s):
                din.copy_(hin, non_blocking=True)
                assert L.prr_linearize(ctx, C.byref(hdr), din.data_ptr(), dout.data_ptr(), n) == 0
                hout.copy_(dout, non_blocking=True)

        for _ in range(3):
            e2e_step()
        s.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        s.synchronize()
        e2e = R.reduce_max(time.perf_counter() - t0)
        e2e = world * args.steps / e2e
    L.prr_ctx_destroy(ctx)
    if rank == 0:
        peak, peak_kind = peaks()
        alg = 4 * n
        achieved = alg / (lin_ms / 1000.0) / 1e9
        line = {
            "metric": "5.8K frames/s linearize", "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": LIN_WORKLOAD, "frames_in_ring": LIN_RING,
                       "l2": "inputs+outputs > L2 (4 x 70 MB ring)", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": "k_linearize", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_value("linearize_5760x3040.md",
                                                                           "traffic_bytes_per_launch"),
                         "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg,
                         "kernel_ms": lin_ms},
            "gpu_launches": int(launches),
        }
        if e2e is not None:
            line["e2e"] = {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": 2 * n, "d2h_bytes_per_step": 2 * n,
                           "note": "pinned host code values in, linear values out, one stream, wall clock"}
        cl = clocks.summary()
        if cl:
            line["clocks"] = cl
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = linearize_cpu(pkts[0], 10.0)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def linearize_cpu(pkt, budget_s: float):
    """The oracle's Frame::linearize on the host cores, frames/s over a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    f = O.decode_frame(pkt, 0, threads)
    f.linearize(threads)
    n, t0 = 0, time.perf_counter()
    while True:
        f.linearize(threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 2000:
            break
    return {"value": n / el, "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": f"{n} linearizations of a {W}x{H} frame, CPU oracle, {threads} threads, {el:.1f} s"}


def run_linearize_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    threads = os.cpu_count() or 1
    f = O.decode_frame(make_packets(1)[0], 0, threads)
    for _ in range(args.warmup):
        f.linearize(threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        f.linearize(threads)
    el = time.perf_counter() - t0
    v = args.steps / el
    line = {
        "impl": "reference", "metric": "5.8K frames/s linearize", "value": v, "unit": "frames/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": LIN_WORKLOAD, "frames_in_ring": LIN_RING},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} linearizations, CPU oracle, {threads} threads"},
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
    ap.add_argument("--workload", default="5k8", choices=["5k8", "mixed-batch", "learned", "8k-stream", "clip", "dng",
                                                               "linearize"],
                    help="5k8: the headline single-frame decode+develop; mixed-batch: 64 uneven frames per step; "
                         "learned: surrogate develop of 4K frames (trains first); 8k-stream: 16 8K frames per step; "
                         "clip: a movie file of 5.8K frames through the clip pipeline, one pass per step; "
                         "dng: 5.8K frames decoded and exported as DNG files (LJ92 tiles on the device); "
                         "linearize: Frame::linearize_into of decoded 5.8K frames")
    ap.add_argument("--epochs", type=int, default=8, help="training epochs for the learned workloads")
    ap.add_argument("--save-model", default="", help="learned: save the trained surrogate (.npz)")
    ap.add_argument("--model", default=os.path.join(ROOT, "proresraw_rs_b200", "data", "surrogate.npz"),
                    help="8k-stream: a trained surrogate (.npz; default the packaged one); trained here if absent")
    ap.add_argument("--batch-frames", type=int, default=BATCH_N, help="mixed-batch: frames per batch")
    ap.add_argument("--no-tune", action="store_true", help="mixed-batch: skip the autotuner (default shape)")
    ap.add_argument("--clip-frames", type=int, default=CLIP_N, help="clip: samples in the movie")
    ap.add_argument("--clip-batch", type=int, default=CLIP_BATCH, help="clip: frames per batch")
    ap.add_argument("--clip-threads", type=int, default=CLIP_THREADS, help="clip: reader threads")
    ap.add_argument("--dng-threads", type=int, default=4, help="dng: host threads of the end-to-end leg")
    ap.add_argument("--overlap", action=argparse.BooleanOptionalAction, default=None,
                    help="5k8 / dng: decode frame k+1 on a second, higher-priority stream while frame k develops "
                         "or is encoded (default: on for 5k8, off for dng, where it was measured slower)")
    ap.add_argument("--develop-ctas", type=int, default=0,
                    help="5k8 --overlap: cap the develop at this many CTAs per SM (0: as many as fit)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--batch-decoders", type=int, default=4,
                    help="decoders taking turns in the mixed-batch end-to-end leg")
    ap.add_argument("--e2e-threads", type=int, default=3,
                    help="host threads (a context each) of the 5k8 end-to-end leg")
    args = ap.parse_args()
    if args.overlap is None:
        args.overlap = args.workload != "dng"
    if args.workload == "mixed-batch":
        return run_batch_reference(args) if args.impl == "reference" else run_batch(args)
    if args.workload == "clip":
        return run_clip_reference(args) if args.impl == "reference" else run_clip(args)
    if args.workload == "dng":
        return run_dng_reference(args) if args.impl == "reference" else run_dng(args)
    if args.workload == "linearize":
        return run_linearize_reference(args) if args.impl == "reference" else run_linearize(args)
    if args.workload in ("learned", "8k-stream"):
        if args.impl == "reference":
            return run_reference(args)
        return run_learned(args) if args.workload == "learned" else run_stream(args)
    if args.impl == "reference":
        return run_reference(args)
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
