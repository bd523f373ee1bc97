#!/usr/bin/env python
"""Benchmark of the two-particle accumulation hot path (G4 measurements per second).

Workload (default "c3"): single-band Hubbard on the 16-site 4x4 cluster, Nw = 64 fermionic
frequencies, all 16 momentum transfers, one frequency transfer, channels PH-magnetic + PH-charge,
per-spin expansion orders n ~ U[50, 400], batches of 64 measurements, synthetic inputs
(dca_b200.workloads).  One step = one batch of 64 measurements through the whole accumulation
(twiddles, NDFT + cluster transform + G, G4 update); G4 (2 x 268 MB FP64) and each batch's G
(1 GB) exceed the 126 MB L2, so no L2 flush is needed between steps.

  value      measurements/s with M already resident in HBM (device pointers), CUDA-event timed;
             each batch's kernels are replayed from the accumulator's CUDA graph of that batch
             shape (captured during the warm-up, which runs at least four batches)
  e2e        the same through the public API with M in pinned host memory (host->device copies
             inside the timed region) and a 4 KiB G4 read-back per step into pinned memory,
             enqueued without blocking (all landed before the clock stops), wall-clock timed;
             value_blocking_readback: the same loop with a blocking read per step
  roofline   the dominant stage, timed with CUDA events on the accumulator's stream around each
             stage's launches, in a second pass over the same steps (eager launches): the
             algorithmic flops (front-end stages) or bytes (G4 update) per launch over
             that time, against the measured dense BF16 peak or HBM copy bandwidth
             (MEASURED_PEAKS.json); update_g4_roofline gives the G4 stage in every run, with the
             DRAM bytes its kernels actually move (committed ncu capture) beside the effective rate
  cpu_baseline  the reference's own CPU TpAccumulator (oracle/_ref/tp_ref_openblas, FP64) on a
             bounded sample: one single-threaded process per core, 1 warm-up and 5 timed
             measurements each, throughput over the wall-clock window of all timed measurements

--impl reference times the reference's CPU accumulator alone (the same workload and unit).
Multi-GPU (torchrun): independent replicas, one per GPU; value = all ranks' measurements / the
slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "G4 meas/s on B200: batched split-BF16 vs plain FP64 at ≤1e-6 rel err; updateG4 HBM %"
UNIT = "meas/s"
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="c3")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison leg")
    p.add_argument("--batch", type=int, default=None, help="measurements per step (default: the workload's)")
    p.add_argument("--nw-half", type=int, default=None,
                   help="positive four-point frequencies (default: the workload's; smaller only for profiling)")
    p.add_argument("--n-range", type=int, nargs=2, default=None, metavar=("LO", "HI"),
                   help="expansion orders per spin (default: the workload's)")
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed",
                   help="path timed as the main leg: the batched mixed path, or the plain FP64 path "
                        "(one measurement at a time; a step is still one batch of measurements)")
    return p.parse_args()


# ------------------------------------------------------------------------------------------------
# Helpers
# ------------------------------------------------------------------------------------------------
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, FALLBACK_BF16_TFLOPS, "fallback"


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons during the timed region.

    NVML is polled from a thread every few milliseconds (read-only queries), so even a timed
    region of a few tens of milliseconds gets samples; nvidia-smi at 200 ms is the fallback."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap",
               "hw_power_brake": "nvmlClocksEventReasonHwPowerBrakeSlowdown"}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, period_s: float = 0.005):
        self.dev = device_index
        self.period = period_s
        self.sm, self.reasons, self.smax = [], set(), None
        self.proc = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.dev)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.lines = []
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _poll(self):
        nv, h = self.nvml
        masks = {k: getattr(nv, v, 0) for k, v in self.REASONS.items()}
        while not self.stop_flag.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for k, m in masks.items():
                    if m and r & m:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(self.period)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.thread.join(timeout=2)
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def workload(args):
    """The named workload with the command line's size overrides (if any) applied."""
    import dataclasses

    from dca_b200 import workloads as W
    w = W.WORKLOADS[args.workload]
    kw = {}
    if args.batch:
        kw["batch"] = args.batch
    if args.nw_half:
        kw["nw_half"] = args.nw_half
        kw["n_sp"] = max(w.n_sp, args.nw_half + w.freq_transfer + 8)
    if args.n_range:
        kw["n_range"] = tuple(args.n_range)
    return dataclasses.replace(w, **kw) if kw else w


def dist_setup(n_gpus):
    from dca_b200 import replicas
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        torch.cuda.set_device(local)
    return replicas.init_from_env("nccl")


def barrier(world):
    from dca_b200 import replicas
    replicas.barrier()


def max_over_ranks(x, world):
    from dca_b200 import replicas
    return replicas.max_over_ranks(x)


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's own TpAccumulator<CPU>, one single-threaded process per core
# ------------------------------------------------------------------------------------------------
def _cpu_workers(per_worker_bytes):
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
        cores = max(1, min(cores, int(avail * 0.6 // per_worker_bytes)))
    except Exception:
        pass
    return max(1, min(cores, 64))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


CPU_WARMUP = 1  # untimed measurements per process (first-touch of the process's G4)
CPU_TIMED = 5   # timed measurements per process


def run_cpu_reference(w, timed, warmup, workers=None):
    """The reference's own TpAccumulator<CPU> (oracle/_ref/tp_ref_openblas, else tp_ref with its
    naive zgemm_, else the restatement oracle) in P single-threaded processes, one per core, each
    accumulating warmup + timed measurements of the workload.  Throughput = all processes' timed
    measurements / the wall-clock window from the first timed measurement's start to the last
    one's end (every process's timed loop lies inside it).  Returns a dict."""
    from dca_b200 import workloads as W
    from oracle import casefile as CF
    from oracle import pyoracle
    cl = w.cluster()
    g0 = W.make_g0(w.model, cl, w.beta, w.chemical_potential(), w.n_sp)
    g4_bytes = 16 * (w.nb ** 4) * cl.nc ** 2 * (2 * w.nw_half) ** 2 * len(w.exchange_momenta(cl.nc)) * len(
        w.exchange_frequencies()) * len(w.channels)
    P = workers or _cpu_workers(g4_bytes * 1.5 + 256e6)
    ref_blas = os.path.join(os.path.dirname(pyoracle.REF_BIN), "tp_ref_openblas")
    binary = ref_blas if os.path.exists(ref_blas) else pyoracle.REF_BIN
    kind = "reference" if os.path.exists(binary) else "port"
    n_per = warmup + timed
    with tempfile.TemporaryDirectory() as d:
        # Every worker's input is written first, then all workers start together, so that their
        # timed loops overlap (the throughput is taken over the union of their windows).
        for i in range(P):
            ms = W.make_measurements(w, n_per, start=10_000 + i * n_per)
            CF.write_case(os.path.join(d, f"w{i}.case"), w, cl, g0, ms)
        procs = []
        for i in range(P):
            case = os.path.join(d, f"w{i}.case")
            out = os.path.join(d, f"w{i}.out")
            if kind == "reference":
                cmd = [binary, case, out, "--no-sp", "--time", "--warmup", str(warmup)]
            else:
                cmd = [sys.executable, "-c",
                       "import sys,time;sys.path.insert(0,%r);from oracle import pyoracle;"
                       "pyoracle.run_case(%r,%r,True,False,warmup=%d,report=True)" % (ROOT, case, out, warmup)]
            env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
            procs.append(subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True,
                                          env=env))
        starts, ends, blas = [], [], "naive-zgemm"
        for pr in procs:
            _, err = pr.communicate()
            if pr.returncode != 0:
                raise RuntimeError(f"CPU baseline worker failed: {err}")
            for tok in err.split():
                k, _, v = tok.partition("=")
                if k == "tp_epoch_start":
                    starts.append(float(v))
                elif k == "tp_epoch_end":
                    ends.append(float(v))
                elif k == "blas":
                    blas = v
    window = max(ends) - min(starts)
    value = P * timed / window
    if kind == "reference":
        blas = ("OpenBLAS (" + blas + ", opencv-python-headless wheel, 1 thread)" if blas != "naive-zgemm"
                else "naive triple-loop zgemm_ (oracle/refbuild/blas_naive.cpp)")
    else:
        blas = "none (restatement, own loops)"
    return {"value": value, "unit": UNIT, "cores": P, "kind": kind,
            "per_core": value / P, "cpu_model": cpu_model(), "blas": blas,
            "sample": f"{P} single-threaded processes (one per core) x {timed} timed {w.name} measurements "
                      f"after {warmup} warm-up, FP64 TpAccumulator<CPU>; window {window:.1f} s from the first "
                      "timed start to the last timed end",
            "window_s": window, "timed_per_process": timed, "warmup_per_process": warmup}


# ------------------------------------------------------------------------------------------------
# Our arm
# ------------------------------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch

    from dca_b200 import workloads as W
    from dca_b200.accumulators import TpAccumulator, TpParameters

    torch.cuda.set_device(local)
    w = workload(args)
    cl = w.cluster()
    g0 = W.make_g0(w.model, cl, w.beta, w.chemical_potential(), w.n_sp)
    B = w.batch
    pool = W.make_measurements(w, 2 * B, start=rank * 1_000_000)
    configs = [list(m.sectors) for m in pool]
    signs = [m.sign for m in pool]
    dev_M = [[torch.from_numpy(np.ascontiguousarray(s.M.T)).cuda().t() for s in m.sectors] for m in pool]
    # Host-resident M for the end-to-end leg: each batch's matrices in one pinned buffer, packed in
    # the order they are accumulated (column major, n x n each), as a caller with a pinned arena
    # per batch holds them; the accumulator then copies a batch in one piece.
    pinned = []
    arenas = []
    for b0 in range(0, len(pool), B):
        mats = [s.M for m in pool[b0:b0 + B] for s in m.sectors]
        arena = torch.empty(max(1, sum(M.shape[0] ** 2 for M in mats)), dtype=torch.float64, pin_memory=True)
        arenas.append(arena)
        flat = arena.numpy()
        off = 0
        for m in pool[b0:b0 + B]:
            pair = []
            for sec in m.sectors:
                n = sec.n
                view = flat[off:off + n * n].reshape(n, n)  # row-major M^T = column-major M
                view[...] = sec.M.T
                pair.append(view.T)
                off += n * n
            pinned.append(pair)

    fp64_main = args.precision == "fp64"
    params = TpParameters.from_workload(w, cl, precision=0 if fp64_main else 1, max_batch=1 if fp64_main else B)
    acc = TpAccumulator(g0, params)
    acc.resetAccumulation(0)
    stream = torch.cuda.ExternalStream(acc.get_stream())

    def step(i, M_src):
        base = (i % 2) * B
        acc.accumulate_batch(M_src[base:base + B], configs[base:base + B], signs[base:base + B])
        acc.flush()

    # Warm-up: at least W batches, until the launch-shape tuner has chosen every tuned launch's
    # shape (each candidate timed three times on real batches) and until both device input sets
    # have their CUDA graph (captured after a batch of the shape ran without tuning probes).
    warmup = 0
    while warmup < args.warmup or ((not acc.tuning_settled() or (acc.graph_stats()[0] < 2 and not fp64_main))
                                   and warmup < 64):
        step(warmup, dev_M)
        warmup += 1
    torch.cuda.synchronize()
    launches0 = acc.kernel_launches()
    graphs0 = acc.graph_stats()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        step(i, dev_M)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1)
    launches = acc.kernel_launches() - launches0
    graphs1 = acc.graph_stats()
    graph_info = {"captured": graphs1[0] - graphs0[0], "batches_replayed": graphs1[1] - graphs0[1]}
    # Stage breakdown: the same steps once more with CUDA events around each stage's launches on
    # the accumulator's stream (eager launches: the events sit between the kernels).
    acc.enable_timing(True)
    for i in range(args.steps):
        step(i, dev_M)
    stages = acc.stage_times()
    acc.enable_timing(False)
    mirror = acc.mirror_mode()
    ms = max_over_ranks(ms_local, world)
    n_meas_total = world * args.steps * B
    value = n_meas_total / (ms / 1e3)

    # End to end through the public API: every step stages a batch whose M sits in pinned host
    # memory (copied to the device inside the timed region, on the accumulator's copy stream) and
    # reads 256 entries of that step's G4 back into pinned host memory.  The reads are enqueued
    # (peek_G4_async), so the next batch is staged and copied while this one computes, the way a
    # solver drives the accumulator; the clock stops after all of them have landed.  The same loop
    # with a blocking read per step is reported beside it.
    res = torch.empty((args.steps, 256), dtype=torch.complex128, pin_memory=True)
    res_np = res.numpy()
    step(0, pinned)  # first host-M batch outside the clock (its first pinned uploads and read-back)
    acc.peek_G4_async(0, 0, res_np[0])
    acc.synchronizeCopy()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(i, pinned)
        acc.peek_G4_async(0, 0, res_np[i])
    acc.synchronizeCopy()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    if not np.array_equal(res_np[-1], acc.peek_G4(0, 0, 256)):
        raise RuntimeError("asynchronous G4 read-back differs from a synchronous one")
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(i, pinned)
        acc.peek_G4(0, 0, 256)
    torch.cuda.synchronize()
    e2e_block_s = max_over_ranks(time.perf_counter() - t0, world)
    h2d = sum(8 * s.n * s.n for m in pool for s in m.sectors) / 2  # mean over the two batches
    e2e = {"value": n_meas_total / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": 256 * 16,
           "readback": "every step, asynchronous into pinned host memory; all landed before the clock stops",
           "value_blocking_readback": n_meas_total / e2e_block_s}
    # The same loop with M in single precision in pinned host memory (a walker run with SpScalar =
    # float hands over float M; dcaacc_tp_accumulate_typed widens it as it is read): half the bytes
    # cross PCIe.  Reported beside the FP64 figure, which stays the headline.
    pinned32, arenas32 = [], []
    if not fp64_main:
        for b0 in range(0, len(pool), B):
            mats = [s.M for m in pool[b0:b0 + B] for s in m.sectors]
            arena = torch.empty(max(1, sum(M.shape[0] ** 2 for M in mats)), dtype=torch.float32, pin_memory=True)
            arenas32.append(arena)
            flat = arena.numpy()
            off = 0
            for m in pool[b0:b0 + B]:
                pair = []
                for sec in m.sectors:
                    n = sec.n
                    view = flat[off:off + n * n].reshape(n, n)
                    view[...] = sec.M.T
                    pair.append(view.T)
                    off += n * n
                pinned32.append(pair)

        def step32(i):
            base = (i % 2) * B
            acc.accumulate_batch_typed(pinned32[base:base + B], configs[base:base + B], signs[base:base + B],
                                       np.float32)
            acc.flush()

        step32(0)  # first host-float batch outside the clock
        acc.synchronizeCopy()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(args.steps):
            step32(i)
            acc.peek_G4_async(0, 0, res_np[i])
        acc.synchronizeCopy()
        torch.cuda.synchronize()
        e2e32_s = max_over_ranks(time.perf_counter() - t0, world)
        e2e["value_fp32_host_m"] = n_meas_total / e2e32_s
        e2e["h2d_bytes_per_step_fp32_host_m"] = int(h2d / 2)

    # Plain FP64, unbatched (the path the mixed one is compared with) and the error between them.
    fp64 = None
    fp64_stages = None
    err = None
    if not args.no_fp64 and not fp64_main:
        n_cmp = B
        ref_acc = TpAccumulator(g0, TpParameters.from_workload(w, cl, precision=0, max_batch=1))
        ref_acc.resetAccumulation(0)
        j = 0
        while j < 2 or (not ref_acc.tuning_settled() and j < 256):  # warm-up, launch shapes tuned
            ref_acc.accumulate(dev_M[j % len(dev_M)], configs[j % len(dev_M)], signs[j % len(dev_M)])
            j += 1
        torch.cuda.synchronize()
        ref_acc.resetAccumulation(0)
        rs = torch.cuda.ExternalStream(ref_acc.get_stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # One call for all measurements (each is still processed on its own, max_batch = 1), so
        # that the host keeps ahead of the GPU.
        e0.record(rs)
        ref_acc.accumulate_batch(dev_M[:n_cmp], configs[:n_cmp], signs[:n_cmp])
        e1.record(rs)
        torch.cuda.synchronize()
        fp64_ms = max_over_ranks(e0.elapsed_time(e1), world)
        fp64 = world * n_cmp / (fp64_ms / 1e3)
        # Stage breakdown in a second pass (events between the kernels).
        ref_acc.resetAccumulation(0)
        ref_acc.enable_timing(True)
        ref_acc.accumulate_batch(dev_M[:n_cmp], configs[:n_cmp], signs[:n_cmp])
        torch.cuda.synchronize()
        fp64_stages = {k: v[0] / n_cmp for k, v in ref_acc.stage_times().items()}
        ref_acc.enable_timing(False)
        ref_acc.finalize()
        # The mixed handle of the timed region, reset, on the same measurements.
        acc.resetAccumulation(1)
        acc.accumulate_batch(dev_M[:n_cmp], configs[:n_cmp], signs[:n_cmp])
        acc.finalize()
        err = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(acc.get_G4(), ref_acc.get_G4())]
        if pinned32:  # and from the single-precision host M of the e2e variant
            acc.resetAccumulation(2)
            acc.accumulate_batch_typed(pinned32[:n_cmp], configs[:n_cmp], signs[:n_cmp], np.float32)
            acc.finalize()
            e2e["rel_err_vs_fp64_fp32_host_m"] = [float(np.linalg.norm(a - b) / np.linalg.norm(b))
                                                  for a, b in zip(acc.get_G4(), ref_acc.get_G4())]
        del ref_acc

    hbm_gbs, bf16_tf, peak_src = peaks()
    simt = os.environ.get("DCAACC_TP_SIMT_ONLY") == "1"
    nc, nb, nw = cl.nc, w.nb, 2 * w.nw_half
    nwe = nw + 2 * w.ext()
    D = nb * nc * nwe
    n_orb = nb * nc
    n_g4 = nb ** 4 * nc ** 2 * nw ** 2 * len(w.exchange_momenta(nc)) * len(w.exchange_frequencies())
    ns = np.array([s.n for m in pool for s in m.sectors], dtype=np.float64)  # both batches of the pool
    per_step = B / len(pool)  # sectors of one step = per_step * (all sectors of the pool)

    # Algorithmic work of each stage, per step (one batch), from the per-spin counts of the reference's
    # two-stage NDFT, cluster transform and G0 products (no dense reformulation credited):
    # row step 8 NwExt n^2 (row NDFT) + 8 Nc D^2 (row half of the cluster transform); column step
    # 8 NwExt^2 n_orb n (column NDFT) + 8 Nc D^2 (column half) + 12 D^2 (G0 epilogue, one band) or
    # 16 nb D^2; G4 update: the FP64 read-modify-write of every running-G4 entry of every channel
    # and one read of the batch's G (FP32 complex, both spins).
    epi = 12.0 if nb == 1 else 16.0 * nb
    alg_flops = {
        "row_transform": per_step * float(np.sum(8.0 * nwe * ns * ns + 8.0 * nc * D * D)),
        "col_transform": per_step * float(np.sum(8.0 * nwe * nwe * n_orb * ns + 8.0 * nc * D * D + epi * D * D)),
    }
    # (plain FP64 path: every measurement reads and writes all of G4 and reads its FP64 G)
    g4_alg_bytes = (B * (len(w.channels) * n_g4 * 32 + 2 * D * D * 16) if fp64_main
                    else len(w.channels) * n_g4 * 32 + B * 2 * D * D * 8)
    g4_sec = stages["update_g4"][0] / args.steps / 1e3  # the stage's time per batch
    g4_paths = {"direct_tc": "discPlanesKernel + frontGemmKernel<2> (disconnected terms) + updateG4DirectMma "
                             "(direct term, G4 flush)",
                "split36": "discPlanesKernel + frontGemmKernel<2> (disconnected terms) + "
                           "updateG4SinglebandOuterSplit (direct term, G4 flush)",
                "staged": "updateG4StagedKernel (all terms, G blocks staged in shared memory)",
                "pp3": "updateG4PPMultibandKernel (particle-particle up-down, 27 band entries per thread)",
                "simt": "updateG4SinglebandBatched",
                "stream": "updateG4SinglebandStream (one measurement, G4 streamed in memory order)",
                "fp64_other": "updateG4SinglebandPH / updateG4Kernel (one measurement)"}
    # Column step and G4 kernels as the accumulator selects them (environment switches included).
    half_any = bool(mirror & 1) or bool(mirror & 2)
    col_env = os.environ.get("DCAACC_TP_FACTORED_COL")
    factorable = nb == 1 and nc == 16 and not fp64_main and not simt
    col_tc = factorable and col_env not in ("0", "1") and os.environ.get("DCAACC_TP_COL_FFT") != "0"
    factored_col = factorable and (col_tc or (col_env == "1" and os.environ.get("DCAACC_TP_COL_FFT") != "0"))
    # 6 x 6 cluster with DCAACC_TP_FACTORED_COL=1: the column step factored on the CUDA cores with the
    # 6 x 6 FFT.
    wide_col = (nb == 1 and nc == 36 and not fp64_main and not simt and col_env == "1"
                and os.environ.get("DCAACC_TP_COL_FFT") != "0")
    factored_col = factored_col or wide_col
    if fp64_main:
        g4_path = "stream" if nb == 1 and nc * nc <= 256 and set(w.channels) <= {2, 3} else "fp64_other"
    elif simt:
        g4_path = "simt"
    elif nb == 3 and tuple(w.channels) == (4,) and not half_any and os.environ.get("DCAACC_TP_PP_GENERIC") != "1":
        g4_path = "pp3"
    elif nb > 1:
        g4_path = "staged"
    elif nc == 36:
        g4_path = "split36"
    else:
        g4_path = "direct_tc"
    stage_kernels = {"update_g4": {"direct_tc": ["discPlanesKernel", "frontGemmKernel<2>", "updateG4DirectMma"],
                                   "split36": ["discPlanesKernel", "frontGemmKernel<2>",
                                               "updateG4SinglebandOuterSplit"],
                                   "staged": ["updateG4StagedKernel"],
                                   "pp3": ["updateG4PPMultibandKernel"],
                                   "stream": ["updateG4SinglebandStream"]}.get(g4_path, []),
                     "col_transform": (["colFactorTcKernel"] if col_tc else ["colFactorWideKernel"] if wide_col else
                                       ["colTwiddlePlanesKernel", "colFactorMmaKernel"] if factored_col
                                       else ["frontGemmKernel<1>"]),
                     "row_transform": ["frontGemmKernel<0>"],
                     "twiddle": (["twiddleWiKernel", "buildMOperandKernel", "buildPhaseOperandKernel"] if factored_col
                                 else ["twiddleWiKernel", "buildMOperandKernel", "buildPhasePairKernel"])}
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of each stage's kernels per launch of
    # the stage, from the committed ncu capture of this workload (cold caches).
    traffic = {}
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            tk = json.load(f)["workloads"].get(w.name + ("-fp64" if fp64_main else ""), {})
        for st, ks in stage_kernels.items():
            if ks and not simt and all(k in tk for k in ks):
                traffic[st] = sum(tk[k]["dram_read_bytes"] + tk[k]["dram_write_bytes"] for k in ks)
    except (OSError, ValueError, KeyError):
        pass

    g4_roof = {"kernels": g4_paths[g4_path], "bound": "hbm",
               "achieved": g4_alg_bytes / g4_sec / 1e9, "peak": hbm_gbs, "unit": "GB/s",
               "frac": g4_alg_bytes / g4_sec / 1e9 / hbm_gbs, "algorithmic_bytes": g4_alg_bytes,
               "ms_per_batch": g4_sec * 1e3, "peak_source": peak_src, "mirror_mode": mirror,
               "frac_of_nominal_8tbs": g4_alg_bytes / g4_sec / 8e12}
    if "update_g4" in traffic:
        # What the kernels actually move (ncu) over the same time: with the mirror symmetry about
        # half of the algorithmic bytes, so this rate is below the effective one above.
        g4_roof["dram_bytes_per_batch"] = traffic["update_g4"]
        g4_roof["dram_gbs"] = traffic["update_g4"] / g4_sec / 1e9
        g4_roof["dram_frac"] = g4_roof["dram_gbs"] / hbm_gbs

    # Roofline of the dominant stage: its algorithmic work per step (one batch) over its kernels'
    # CUDA-event time per step (the stage's launches: one per batch for the tensor-core GEMMs, one
    # per measurement on the plain FP64 path).
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms, dom_launches = stages[dom]
    per_launch_ms = dom_ms / args.steps
    sec = per_launch_ms / 1e3
    tc_front = not simt and not fp64_main
    if dom == "update_g4":
        roof = {"kernel": "update_g4 stage: " + g4_roof["kernels"], "bound": "hbm",
                "achieved": g4_alg_bytes / sec / 1e9, "peak": hbm_gbs, "unit": "GB/s",
                "algorithmic_bytes": g4_alg_bytes}
        for k in ("dram_gbs", "dram_frac"):
            if k in g4_roof:
                roof[k] = g4_roof[k]
    elif dom in ("col_transform", "row_transform") and tc_front:
        # Tensor-core front-end: the algorithmic flops against the measured dense BF16 peak.
        # Beside it, the work the kernel is built to do (the dense complex product over all vertices,
        # split FP16: three MMAs per complex multiply-add pair) and its issued MMA rate (128 x 128
        # tiles, K padded to 32) against the same peak.
        chunks = np.ceil(ns / 32)
        Dp = -(-D // 128) * 128
        mma_flop = 2.0 * 128 * 128 * 16
        rows_done = 0.5 if mirror & 1 else 1.0  # half G: the upper frequency half of the rows
        if dom == "col_transform" and factored_col:
            # The orbital-factored column step (no dense product): its work is the algorithmic one
            # (plus the site-masked zeros of its MMAs), so only the algorithmic rate is reported.
            dense = mma = None
            kern = ("colFactorTcKernel (column step factored by orbital: per-site sums in tensor memory, "
                    "4 x 4 FFT, G0 factor)" if col_tc else
                    "colFactorWideKernel (column step factored by orbital on the CUDA cores, 6 x 6 FFT, G0 factor)"
                    if wide_col else "colTwiddlePlanesKernel + colFactorMmaKernel (orbital-factored column step)")
        elif dom == "col_transform":
            dense = per_step * float(np.sum(8.0 * D * D * ns)) * rows_done
            mma = per_step * float(np.sum((Dp // 128) ** 2 * rows_done * chunks * 24 * mma_flop))
            kern = "frontGemmKernel<1> (column step, G = X' Q^H + beta G0 delta)"
        else:
            dense = per_step * float(np.sum(4.0 * D * ns * ns)) * rows_done
            mma = per_step * float(np.sum((Dp // 128) * rows_done * np.ceil(ns / 128) * chunks * 12 * mma_flop))
            kern = "frontGemmKernel<0> (row step, X' = P M)"
        roof = {"kernel": kern, "bound": "tensor", "achieved": alg_flops[dom] / sec / 1e12, "peak": bf16_tf,
                "unit": "TFLOP/s", "algorithmic_flops": alg_flops[dom],
                "peak_note": "measured dense BF16 burst peak; algorithmic flops per spin of the reference's "
                             "two-stage form, so the dense reformulation's extra work is not credited",
                }
        if dense is not None:
            roof.update({"dense_form_flops": dense, "dense_form_tflops": dense / sec / 1e12,
                         "mma_issued_tflops": mma / sec / 1e12, "mma_frac_of_bf16_peak": mma / sec / 1e12 / bf16_tf})
        else:
            roof["work_note"] = ("factored by orbital: the column NDFT per site on the CUDA cores (FP32), then the "
                                 "6 x 6 FFT over the sites; no dense product" if wide_col else
                                 "factored by orbital: the column NDFT per site on the tensor cores, then the 4 x 4 "
                                 "FFT over the sites; no dense product")
            # The same stage against HBM: it must read X' (four FP16 planes, 8 bytes per complex
            # entry) and write G (FP32 complex) once, for the rows it computes.
            mem_bytes = per_step * rows_done * float(np.sum(D * ns * 8.0 + D * D * 8.0))
            roof["memory_view"] = {"algorithmic_bytes": mem_bytes, "achieved_gbs": mem_bytes / sec / 1e9,
                                   "frac_of_hbm": mem_bytes / sec / 1e9 / hbm_gbs,
                                   "note": "X' read and G written once per launch, for the rows computed"}
    else:
        # SIMT front-end stages are dominated by their global traffic (M / X' / G, complex of the
        # path's precision).
        mean_n = float(np.mean(ns))
        cs = 16 if fp64_main else 8
        real = "double" if fp64_main else "float"
        if dom == "col_transform":
            alg_bytes = 2 * B * (D * mean_n * cs + D * D * cs)
            kern = f"colTransformKernel<{real}>"
        elif dom == "row_transform":
            alg_bytes = 2 * B * (mean_n * mean_n * 8 + D * mean_n * cs)
            kern = f"rowTransformKernel<{real}>"
        else:
            alg_bytes = 2 * B * mean_n * nwe * 16
            kern = "twiddleKernel"
        roof = {"kernel": kern, "bound": "hbm", "achieved": alg_bytes / sec / 1e9,
                "peak": hbm_gbs, "unit": "GB/s"}
    roof["frac"] = roof["achieved"] / roof["peak"]
    roof["peak_source"] = peak_src + " (MEASURED_PEAKS.json)" if peak_src == "measured" else peak_src
    roof["ms_per_step"] = per_launch_ms
    roof["launches_per_step"] = dom_launches / args.steps
    roof["traffic"] = traffic.get(dom)
    if roof["traffic"] is not None:
        roof["traffic_unit"] = "DRAM bytes per launch of the stage (ncu, profiles/dram_traffic.json)"
    stage_frac = {}
    for st, (ms_st, _n) in stages.items():
        t_st = ms_st / args.steps / 1e3
        if st in alg_flops:
            stage_frac[st] = {"tflops": alg_flops[st] / t_st / 1e12, "frac_of_bf16": alg_flops[st] / t_st / 1e12 / bf16_tf}
        elif st == "update_g4":
            stage_frac[st] = {"gbs": g4_alg_bytes / t_st / 1e9, "frac_of_hbm": g4_alg_bytes / t_st / 1e9 / hbm_gbs}

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "fp64" if fp64_main else "fp32 (G, G4 partials) + fp64 (running G4)",
        "data": "synthetic (seeded; dca_b200.workloads)",
        "config": bench_config(w, world),
        "warmup_batches_run": warmup,
        "warmup_note": "untimed batches: at least --warmup, and on until the launch-shape tuner has settled "
                       "and both CUDA graphs exist",
        "measurements_per_step": B, "precision": args.precision,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "cuda_graphs": graph_info,
        "launch_tuning": [line for line in acc.tuning_report().splitlines() if line],
        "mirror_mode": {"half_g": bool(mirror & 1), "half_g4": bool(mirror & 2)},
        "roofline": roof,
        "update_g4_roofline": g4_roof,
        "stages_ms_per_step": {k: v[0] / args.steps for k, v in stages.items()},
        "stages_roofline": stage_frac,
        "fp64_unbatched_meas_per_s": fp64,
        "fp64_stages_ms_per_meas": fp64_stages,
        "speedup_vs_fp64": (value / fp64) if fp64 else None,
        "rel_err_vs_fp64": err,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = run_cpu_reference(w, CPU_TIMED, CPU_WARMUP)
        # The reference's own scale (2x2 cluster, c1) at one core and at all cores.
        c1 = W.WORKLOADS["c1"]
        one = run_cpu_reference(c1, 200, 5, workers=1)
        allc = run_cpu_reference(c1, 200, 5)
        result["cpu_baseline"]["c1"] = {"workload": c1.describe(with_batch=False),
                                        "one_core": one["value"], "all_cores": allc["value"],
                                        "cores": allc["cores"], "unit": UNIT}
    return result


def bench_config(w, world):
    """The workload both arms measure (the same dict in both lines): the configuration with its
    batch, how the GPU arm spreads it, and its data sizes against L2."""
    cl = w.cluster()
    nwe = 2 * w.nw_half + 2 * w.ext()
    D = w.nb * cl.nc * nwe
    n_g4 = w.nb ** 4 * cl.nc ** 2 * (2 * w.nw_half) ** 2 * len(w.exchange_momenta(cl.nc)) * len(w.exchange_frequencies())
    g4_mb, g_gb = len(w.channels) * n_g4 * 16 / 1e6, w.batch * 2 * D * D * 8 / 1e9
    big = g4_mb + 1e3 * g_gb > 126.0
    return {"workload": w.describe(), "parallelism": f"replicas x{world}",
            "l2": f"inputs {'larger' if big else 'smaller'} than L2 (G4 {g4_mb:.0f} MB, G {g_gb:.1f} GB per batch)"
                  + ("" if big else "; L2 is not flushed between steps")}


def run_reference_arm(args, world, rank):
    """The reference's CPU accumulator on the host cores: one step = one measurement in each of the
    P processes.  The run is bounded to a few minutes (about 3 s per c3 measurement and core): at
    most 5 warm-up and 20 timed steps, and the line reports the steps actually run."""
    from dca_b200 import workloads as W
    w = workload(args)
    if rank != 0:
        return None
    timed = max(1, min(args.steps, 20))
    warm = min(args.warmup, 5)
    cb = run_cpu_reference(w, timed, warm)
    val = cb["value"]
    return {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
            "steps": timed, "warmup": warm, "steps_requested": args.steps,
            "ms_per_step": 1e3 * cb["window_s"] / timed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded; dca_b200.workloads)",
            "config": bench_config(w, world),
            "parallelism": f"{cb['cores']} CPU processes, one per core, one measurement at a time each",
            "cpu_baseline": cb,
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse_args()
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            res = run_reference_arm(args, world, rank)
        else:
            res = run_ours(args, world, rank, local)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
