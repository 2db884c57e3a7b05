#!/usr/bin/env python
"""MANS compress/decompress throughput on B200 (one JSON line on rank 0).

A step is one compress + one decompress of one buffer, bit-exact. Default
workload: 16 frames of 4096 x 4096 uint32 detector data (1 GiB; Gamma(0.5,20)
background, 0.1% peaks in [1e4, 1e6]), synthetic and seeded. Inputs are far
larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl mans|reference]
                  [--workload detector_u32|laplace_u16|volume_u16]

N > 1 (launched by torchrun): every rank runs an independent replica on its
own GPU (the codec has no cross-buffer exchange), timing is the max over
ranks and the value is the whole job's bytes over that time (weak scaling).

--impl reference times the reference's CPU implementation of the path on the
host cores instead (rank 0 only): the reference's own CPU mapping
(mapping/cpu/mappingcpuV2.cpp, built under oracle/_ref) where it exists
(uint16) and the C port of the rest (the reference has no CPU rANS and no
CPU uint32 mapping).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "compress/decompress GB/s on 1 B200 (bit-exact); batched vs plain; p50/p99 latency"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "detector_u32": dict(n=16 * 4096 * 4096, dtype="uint32",
                         desc="detector_u32: 16 frames x 4096 x 4096 uint32 (1 GiB), "
                              "round(Gamma(0.5, 20)) + 0.1% uniform peaks in [1e4, 1e6]"),
    "laplace_u16": dict(n=4_194_304, dtype="uint16",
                        desc="laplace_u16: 4,194,304 uint16 (8 MiB), round(32768 + Laplace(0, 40))"),
    "volume_u16": dict(n=2048 * 2048 * 256, dtype="uint16",
                       desc="volume_u16: 2048 x 2048 x 256 uint16 (2 GiB), N(20000,3000) rows + N(0,150)"),
    "gradient_u16": dict(n=1 << 29, dtype="uint16",
                         desc="gradient_u16: 2^29 uint16 (1 GiB), one buffer of the mixed workload's "
                              "uint16 kind: 8000 + a*x/1024 + b*y/H + N(0, 200)"),
    "quant_u32": dict(n=1 << 28, dtype="uint32",
                      desc="quant_u32: 2^28 uint32 (1 GiB), one buffer of the mixed workload's "
                           "uint32 kind: 2^31 + round(Laplace(0, 300))"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mans", "reference"], default="mans")
    ap.add_argument("--workload", choices=list(WORKLOADS) + ["mixed_c3", "serve_c5"],
                    default="detector_u32")
    ap.add_argument("--requests", type=int, default=0, help="serve_c5: requests (100000)")
    ap.add_argument("--corpus", type=int, default=0, help="serve_c5: distinct buffers (256)")
    ap.add_argument("--rate", type=float, default=20.0, help="serve_c5: offered GB/s")
    ap.add_argument("--saturation-requests", type=int, default=4000)
    ap.add_argument("--no-check", action="store_true", help="serve_c5: skip the per-result check")
    ap.add_argument("--items", type=int, default=0, help="mixed_c3: number of buffers (4096)")
    ap.add_argument("--merged-ratio", type=int, default=120,
                    help="mixed_c3: mapped-byte room per buffer, percent of its bytes")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--precision", type=int, default=10)
    ap.add_argument("--n", type=int, default=0, help="override the element count (profiling runs)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true",
                    help="mixed_c3: skip the end-to-end pass through host buffers")
    ap.add_argument("--no-sub", action="store_true",
                    help="default workload: skip the mixed_c3 / serve_c5 / reference_gpu sub-records")
    ap.add_argument("--sub-steps", type=int, default=3, help="mixed_c3 sub-record: timed steps")
    ap.add_argument("--sub-requests", type=int, default=20_000,
                    help="serve_c5 sub-record: requests of the Poisson trace")
    ap.add_argument("--traffic-json", default=os.path.join(ROOT, "profiles", "dram_traffic.json"),
                    help="ncu-measured DRAM bytes per launch of each kernel (roofline.traffic)")
    ap.add_argument("--no-check-oracle", action="store_true",
                    help="skip the comparison of the whole stream with the multi-threaded "
                         "oracle (run after the timed region)")
    return ap.parse_args()


# ---------------------------------------------------------------- data
from mans_b200.workloads import gen_device, gen_mixed_device  # noqa: E402


def gen_host_sample(workload: str, n: int, seed: int) -> np.ndarray:
    from mans_b200 import workloads as W
    if workload == "detector_u32":
        return W.detector_u32(n, seed)
    if workload == "laplace_u16":
        return W.laplace_u16(n, seed)
    if workload == "gradient_u16":
        return W.gradient_u16(n, seed)
    if workload == "quant_u32":
        return W.quant_u32(n, seed)
    return W.volume_u16(n, seed)


# ---------------------------------------------------------------- clocks (NVML)
class ClockSampler:
    """Samples SM clock, power and clock-event reasons every ~10 ms via NVML."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4,
        "hw_slowdown": 0x8, "sync_boost": 0x10, "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80,
        "display_clock_setting": 0x100,
    }

    def __init__(self, device_index: int):
        self.samples = []
        self.ok = False
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self._reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.ok = True
        except Exception as e:  # pragma: no cover - depends on the box
            self.err = str(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                clk = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = self._reasons(self.h)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.samples.append((clk, rs, pw))
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self) -> dict:
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": getattr(self, "max_mhz", None), "reasons": [],
                    "samples": 0}
        clks = [s[0] for s in self.samples]
        mask = 0
        for s in self.samples:
            mask |= s[1]
        reasons = [k for k, v in self.REASONS.items() if mask & v and k != "gpu_idle"]
        return {"sm_mhz": statistics.median(clks), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(clks), "power_w_max": round(max(s[2] for s in self.samples), 1)}


# ---------------------------------------------------------------- helpers
def hbm_peak() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def measured_traffic(path: str, workload: str, n: int) -> dict:
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum)
    of each kernel, as measured by ncu on this workload at this size and
    recorded in a JSON data file: {workload: {"n": elements, "kernels":
    {kernel: bytes}}}. Empty when the file holds no record for (workload, n)."""
    try:
        with open(path) as f:
            rec = json.load(f).get(workload, {})
    except (OSError, ValueError):
        return {}
    return {k: int(v) for k, v in rec.get("kernels", {}).items()} if rec.get("n") == n else {}


def reduce_max_over_ranks(values, dist=None, device="cuda"):
    """Max of each value over the ranks (the job's timing is its slowest rank)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- CPU timing (reference arm / baseline)
def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_round_trip(workload: str, n: int, reps: int, warm: int, seed: int = 7) -> dict:
    """Round trip of a host sample through the CPU path on all host cores,
    plus a one-thread figure on a sixteenth of the sample."""
    x = gen_host_sample(workload, n, seed)
    r = cpu_round_trip_array(x, reps, warm, f"the same generator, seed {seed}")
    x1 = x[: max(1, (x.size // 16) // 512 * 512)]
    r1 = cpu_round_trip_array(x1, 3, 1, f"the same generator, seed {seed}", threads=1)
    r["one_thread"] = {"value": r1["value"], "unit": r1["unit"], "sample": r1["sample"]}
    return r


def cpu_round_trip_array(x: np.ndarray, reps: int, warm: int, what: str,
                         threads: int = 0) -> dict:
    from oracle import pyoracle as O
    n = x.size
    L = O.lib()
    u8p, u16p, u32p = O.u8p, O.u16p, O.u32p
    cores = threads or os.cpu_count() or 1
    L.mo_set_threads(cores)
    times = []
    kind = "port"
    detail = ""
    if x.dtype == np.uint32:
        cap = L.mo_adm_u32_max_merged_size(n)
        m = np.empty(cap, np.uint8)
        back = np.empty(n, np.uint32)
        scratch_words = L.mo_ans_par_scratch_words(cap)
        scratch = np.empty(max(scratch_words, 1), np.uint16)
        sst = np.empty(max(32 * ((cap + 4095) // 4096), 1), np.uint32)
        snw = np.empty(max((cap + 4095) // 4096, 1), np.uint32)
        scap = O.max_compressed_size(cap)
        s = np.empty(scap, np.uint8)
        mb = np.empty(cap, np.uint8)
        detail = ("ADM uint32 escape mapping and byte rANS: C port (oracle/mans_oracle.c, OpenMP); "
                  "the reference has no CPU implementation of either")
        for it in range(warm + reps):
            t0 = time.perf_counter()
            msize = L.mo_adm_u32_map_par(x.ctypes.data_as(u32p), n, m.ctypes.data_as(u8p), cap)
            ssize = L.mo_ans_encode_par(10, m.ctypes.data_as(u8p), msize, s.ctypes.data_as(u8p), scap,
                                        scratch.ctypes.data_as(u16p), sst.ctypes.data_as(u32p),
                                        snw.ctypes.data_as(u32p))
            L.mo_ans_decode_par(s.ctypes.data_as(u8p), ssize, mb.ctypes.data_as(u8p), cap)
            L.mo_adm_u32_unmap_par(mb.ctypes.data_as(u8p), msize, n, back.ctypes.data_as(u32p))
            dt = time.perf_counter() - t0
            if it >= warm:
                times.append(dt)
        ok = bool(np.array_equal(back, x))
    else:
        R = O.ref_lib()
        ref = O.RefAdmCpu(x, threads=cores) if R is not None else None
        ms_cap = 6 * ((n + 511) // 512) + n + 64 * n  # generous
        m = np.empty(ms_cap, np.uint8)
        scap = O.max_compressed_size(ms_cap)
        s = np.empty(scap, np.uint8)
        scratch = np.empty(max(L.mo_ans_par_scratch_words(ms_cap), 1), np.uint16)
        sst = np.empty(32 * ((ms_cap + 4095) // 4096), np.uint32)
        snw = np.empty((ms_cap + 4095) // 4096, np.uint32)
        mb = np.empty(ms_cap, np.uint8)
        if ref is not None:
            kind = "reference"
            detail = ("ADM uint16: the reference's mapping/cpu/mappingcpuV2.cpp (OpenMP); byte rANS: "
                      "C port (the reference has no CPU rANS)")
        for it in range(warm + reps):
            t0 = time.perf_counter()
            if ref is not None:
                ref.compress()
                mm = ref.merged(True)
                msize = mm.size
                msrc = mm
            else:
                msrc = O.adm_u16_map(x)
                msize = msrc.size
            ssize = L.mo_ans_encode_par(10, msrc.ctypes.data_as(u8p), msize, s.ctypes.data_as(u8p),
                                        scap, scratch.ctypes.data_as(u16p), sst.ctypes.data_as(u32p),
                                        snw.ctypes.data_as(u32p))
            L.mo_ans_decode_par(s.ctypes.data_as(u8p), ssize, mb.ctypes.data_as(u8p), ms_cap)
            if ref is not None:
                ref.decompress()
            else:
                O.adm_u16_unmap(mb[:msize], n)
            dt = time.perf_counter() - t0
            if it >= warm:
                times.append(dt)
        ok = True
    mean = sum(times) / len(times)
    nbytes = n * x.itemsize
    return {"value": round(nbytes / mean / 1e9, 4), "unit": "GB/s", "cores": cores, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": f"{n} elements ({nbytes / 1e6:.1f} MB) of {what}; "
                      f"mean of {reps} round trips after {warm} warm-ups; {detail}",
            "round_trip_ok": ok, "ms_per_round_trip": round(mean * 1e3, 3)}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    steps = max(1, args.steps)
    warm = max(0, args.warmup)
    if args.workload == "mixed_c3":
        cb = mixed_cpu_sample(steps, warm)
        line = {
            "metric": METRIC, "value": cb["value"], "unit": "GB/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": cb["ms_per_round_trip"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16+u32",
            "data": "synthetic",
            "config": {"workload": MIXED_DESC.format(count=args.items or 4096), "precision": 10},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    wl = WORKLOADS[args.workload]
    n_sample = {"detector_u32": 1 << 24, "laplace_u16": wl["n"], "volume_u16": 1 << 25,
                    "gradient_u16": 1 << 25, "quant_u32": 1 << 24}[args.workload]
    cb = cpu_round_trip(args.workload, n_sample, steps, warm)
    line = {
        "metric": METRIC, "value": cb["value"], "unit": "GB/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": cb["ms_per_round_trip"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32" if wl["dtype"] == "uint32" else "u16", "data": "synthetic",
        "config": {"workload": wl["desc"], "sample_elems": n_sample, "precision": 10},
        "impl": "reference", "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def run_mans(args):
    import torch

    import mans_b200 as mb

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    wl = WORKLOADS[args.workload]
    n = args.n or wl["n"]
    x = gen_device(args.workload, n, seed=2 + rank)
    elem = x.element_size()
    U = n * elem
    code = mb.dtype_code(x)
    ws = mb.Workspace(U)
    cap = mb.max_compressed_size(code, n)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    back = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    def step():
        mb.compress_into(ws, x, out, size, args.precision, stream)
        mb.decompress_into(ws, out, cap, back, stream)

    for _ in range(max(3, args.warmup)):
        step()
    ws.check(stream, "warm-up")
    C = int(size.item())
    hdr = out[:32].cpu().numpy().view(np.uint32)
    M = int(hdr[2])  # mapped bytes = rANS uncompressed size recorded in the stream
    bit_exact = bool(torch.equal(back.view(torch.uint8), x.view(torch.uint8)))

    # ---- timed region (device events, max over ranks)
    ws.set_timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    kt = ws.kernel_times()
    ws.set_timing(False)
    ws.check(stream, "timed steps")
    bit_exact = bit_exact and bool(torch.equal(back.view(torch.uint8), x.view(torch.uint8)))
    kcalls = max(1, kt["compress_calls"])
    dcalls = max(1, kt["decompress_calls"])
    k_ms = {"map": kt["map"] / kcalls, "encode": kt["encode"] / kcalls,
            "decode": kt["decode"] / dcalls, "unmap": kt["unmap"] / dcalls}
    comp_ms = k_ms["map"] + k_ms["encode"]
    decomp_ms = k_ms["decode"] + k_ms["unmap"]

    ms_total, comp_ms, decomp_ms = reduce_max_over_ranks([ms_total, comp_ms, decomp_ms], dist)
    ms_step = ms_total / args.steps
    value = world * U * args.steps / (ms_total / 1e3) / 1e9

    # ---- end to end through the public API with host buffers
    # (a) one buffer at a time: H2D input, compress, D2H stream, H2D stream,
    #     decompress, D2H values, then the next buffer;
    # (b) a sequence of buffers pipelined over two streams, each with its
    #     own device buffers: PCIe is full duplex, so one step's downloads
    #     run under the next steps' uploads. Every step's own copies are
    #     inside the timed region in both.
    h_in = torch.empty(U, dtype=torch.uint8, pin_memory=True)
    h_in.copy_(x.view(torch.uint8))
    scap = C + 4096
    e2e_seq_ms = []
    sets = []
    depth = int(os.environ.get("MANS_E2E_DEPTH", "2"))  # buffer sets in flight
    for i in range(depth):
        wsi = ws if i == 0 else mb.Workspace(U)
        sets.append({
            "ws": wsi, "s": stream if i == 0 else torch.cuda.Stream(),
            "d_in": torch.empty_like(x), "out": out if i == 0 else torch.empty(cap, dtype=torch.uint8, device="cuda"),
            "size": size if i == 0 else torch.zeros(1, dtype=torch.int64, device="cuda"),
            "d_s": torch.empty(scap, dtype=torch.uint8, device="cuda"), "d_back": torch.empty_like(x),
            "h_s": torch.empty(scap, dtype=torch.uint8, pin_memory=True),
            "h_size": torch.empty(1, dtype=torch.int64, pin_memory=True),
            "h_out": torch.zeros(U, dtype=torch.uint8, pin_memory=True),
            "ev": torch.cuda.Event()})

    # Each buffer set has an upload, a download and a kernel stream, so that
    # a set's next upload overlaps its previous download and no copy waits
    # behind another set's copies. Events order every use of a set's buffers
    # after the previous use is finished.
    for S in sets:
        S["up"], S["down"] = torch.cuda.Stream(), torch.cuda.Stream()
        for e in ("e_in", "e_c", "e_size", "e_sd", "e_su", "e_dc", "e_free"):
            S[e] = torch.cuda.Event()

    def first_half(S):
        S["up"].wait_event(S["e_c"])  # the set's previous compress has read d_in
        with torch.cuda.stream(S["up"]):
            S["d_in"].view(torch.uint8).copy_(h_in, non_blocking=True)
            S["e_in"].record(S["up"])
        S["s"].wait_event(S["e_in"])
        S["s"].wait_event(S["e_free"])  # the previous step's out / d_back are read
        mb.compress_into(S["ws"], S["d_in"], S["out"], S["size"], args.precision, S["s"])
        S["e_c"].record(S["s"])
        S["down"].wait_event(S["e_c"])
        with torch.cuda.stream(S["down"]):
            S["h_size"].copy_(S["size"], non_blocking=True)
            S["e_size"].record(S["down"])

    def second_half(S):
        S["e_size"].synchronize()  # the compressed size, read on the host
        c = int(S["h_size"].item())
        with torch.cuda.stream(S["down"]):
            S["h_s"][:c].copy_(S["out"][:c], non_blocking=True)
            S["e_sd"].record(S["down"])
        S["up"].wait_event(S["e_sd"])
        with torch.cuda.stream(S["up"]):
            S["d_s"][:c].copy_(S["h_s"][:c], non_blocking=True)
            S["e_su"].record(S["up"])
        S["s"].wait_event(S["e_su"])
        mb.decompress_into(S["ws"], S["d_s"], c, S["d_back"], S["s"])
        S["e_dc"].record(S["s"])
        S["down"].wait_event(S["e_dc"])
        with torch.cuda.stream(S["down"]):
            S["h_out"].copy_(S["d_back"].view(torch.uint8), non_blocking=True)
            S["e_free"].record(S["down"])

    cur = torch.cuda.current_stream()
    for it in range(1 + args.e2e_steps):  # (a)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(cur)
        for st_ in (sets[0]["up"], sets[0]["down"], sets[0]["s"]):
            st_.wait_stream(cur)
        first_half(sets[0])
        second_half(sets[0])
        for st_ in (sets[0]["up"], sets[0]["down"], sets[0]["s"]):
            cur.wait_stream(st_)
        b.record(cur)
        torch.cuda.synchronize()
        if it > 0:
            e2e_seq_ms.append(a.elapsed_time(b))
    e2e_ok = bool(torch.equal(sets[0]["h_out"], h_in))
    # (b): one untimed warm-up round, then the timed sequence; long enough
    # that filling and draining the pipeline (one step's full chain of
    # copies and kernels) is a small part of the time per step
    n_pipe = max(16, 4 * args.e2e_steps)
    for timed in (False, True):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(cur)
        for st_ in [x for S in sets for x in (S["up"], S["down"], S["s"])]:
            st_.wait_stream(cur)
        steps_here = n_pipe if timed else depth
        pending = []
        for k in range(steps_here):
            S = sets[k % depth]
            first_half(S)
            pending.append(S)
            if len(pending) == depth:  # the oldest step's second half
                second_half(pending.pop(0))
        while pending:
            second_half(pending.pop(0))
        for st_ in [x for S in sets for x in (S["up"], S["down"], S["s"])]:
            cur.wait_stream(st_)
        b.record(cur)
        torch.cuda.synchronize()
    e2e_pipe_ms = a.elapsed_time(b) / n_pipe
    for S in sets:
        S["ws"].check(S["s"], "e2e")
        e2e_ok = e2e_ok and bool(torch.equal(S["h_out"], h_in))
    for S in sets[1:]:
        S["ws"].close()
    e2e_step_ms, e2e_seq_step_ms = reduce_max_over_ranks(
        [e2e_pipe_ms, sum(e2e_seq_ms) / len(e2e_seq_ms)], dist)

    result = None
    if rank == 0:
        peak, peak_src = hbm_peak()
        algo = {"map": U + M, "encode": M + C, "decode": C + M, "unmap": M + U}
        names = {"map": "adm_u32_map_kernel" if elem == 4 else "adm_u16_map_kernel",
                 "encode": "ans_encode_kernel", "decode": "ans_decode_kernel",
                 "unmap": "adm_u32_unmap_kernel" if elem == 4 else "adm_u16_unmap_kernel"}
        dom = max(k_ms, key=lambda k: k_ms[k])
        achieved = algo[dom] / (k_ms[dom] / 1e3) / 1e9
        traffic = measured_traffic(args.traffic_json, args.workload, n).get(names[dom])
        kernels = {names[k]: {"ms": round(k_ms[k], 4), "algorithmic_bytes": algo[k],
                              "gbs": round(algo[k] / (k_ms[k] / 1e3) / 1e9, 1) if k_ms[k] else None,
                              "frac_of_hbm": round(algo[k] / (k_ms[k] / 1e3) / 1e9 / peak, 4) if k_ms[k] else None}
                   for k in k_ms}
        result = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32" if elem == 4 else "u16", "data": "synthetic",
            "config": {"workload": (wl["desc"] if n == wl["n"] else f"{args.workload} with n={n}")
                       + "; one buffer, compress + decompress per step",
                       "n_elems": n, "uncompressed_bytes": U, "precision": args.precision,
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "compress_gbs": round(U / (comp_ms / 1e3) / 1e9, 2),
            "decompress_gbs": round(U / (decomp_ms / 1e3) / 1e9, 2),
            "compressed_bytes": C, "mapped_bytes": M, "compression_ratio": round(U / C, 4),
            "bit_exact_round_trip": bit_exact and e2e_ok,
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": round(achieved, 1),
                         "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic},
            "kernels": kernels,
            "e2e": {"value": round(world * U / (e2e_step_ms / 1e3) / 1e9, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": U + C, "d2h_bytes_per_step": 8 + C + U,
                    "ms_per_step": round(e2e_step_ms, 3),
                    "mode": f"{n_pipe} buffers pipelined over {depth} buffer sets, each with upload, download and kernel streams"},
            "e2e_sequential": {"value": round(world * U / (e2e_seq_step_ms / 1e3) / 1e9, 3),
                               "unit": "GB/s", "ms_per_step": round(e2e_seq_step_ms, 3),
                               "mode": "one buffer at a time"},
            "gpu_launches": 4 * args.steps,
            "clocks": clk.summary(),
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ws.close()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            n_sample = {"detector_u32": 1 << 24, "laplace_u16": n, "volume_u16": 1 << 25,
                        "gradient_u16": 1 << 25, "quant_u32": 1 << 24}[args.workload]
            result["cpu_baseline"] = cpu_round_trip(args.workload, n_sample, reps=5, warm=2)
        if not args.no_check_oracle:
            t0 = time.time()
            result["oracle_stream_equal"] = check_oracle(args, x, out[:C])
            result["oracle_check"] = {
                "what": "the whole compressed stream of the benchmarked input, byte for byte, "
                        "against the oracle's group- and block-parallel restatement "
                        "(oracle/mans_oracle.c), after the timed region",
                "seconds": round(time.time() - t0, 1)}
    return result


# ---------------------------------------------------------------- mixed batch
MIXED_DESC = ("mixed_c3: {count} buffers, sizes log-uniform in [4 KiB, 64 MiB] rounded down to 1 KiB "
              "(seed 3), alternating uint16 gradients (8000 + a*x/1024 + b*y/H + N(0, 200), "
              "a, b ~ U(-1000, 1000)) and uint32 quantisation codes (2^31 + round(Laplace(0, 300)))")


def mixed_layout(count: int, seed: int = 3):
    """Buffers of the mixed workload: element size, count, bytes, 256-byte aligned offset."""
    from mans_b200 import workloads as W
    sizes = W.mixed_sizes(count, seed)
    ab = np.random.default_rng(seed + 100).uniform(-1000, 1000, (count, 2))
    items, off = [], 0
    for i, nb in enumerate(sizes.tolist()):
        elem = 2 if i % 2 == 0 else 4
        items.append({"elem": elem, "n": nb // elem, "bytes": nb // elem * elem, "off": off,
                      "a": float(ab[i, 0]), "b": float(ab[i, 1])})
        off += (nb + 255) // 256 * 256
    return items, off


def mixed_cpu_sample(reps: int, warm: int) -> dict:
    """CPU round trip of one buffer of each kind of the mixed workload (16 MB each)."""
    from mans_b200 import workloads as W
    parts = [cpu_round_trip_array(W.gradient_u16(1 << 23, 7), reps, warm, "uint16 gradient"),
             cpu_round_trip_array(W.quant_u32(1 << 22, 7), reps, warm, "uint32 Laplace+2^31")]
    nbytes = 2 * (16 << 20)
    t = sum(p["ms_per_round_trip"] for p in parts) / 1e3
    return {"value": round(nbytes / t / 1e9, 4), "unit": "GB/s", "cores": parts[0]["cores"],
            "kind": parts[0]["kind"] if parts[0]["kind"] == parts[1]["kind"] else "reference+port",
            "sample": "one 16 MB buffer of each kind of the mixed workload: "
                      + " | ".join(p["sample"] for p in parts),
            "round_trip_ok": all(p["round_trip_ok"] for p in parts),
            "ms_per_round_trip": round(t * 1e3, 3)}


def run_mixed(args):
    """Batched vs plain on the mixed workload: every buffer compressed and
    decompressed once per step, (a) through one batched call per direction
    replayed from a CUDA graph and (b) through one plain call per buffer."""
    import torch

    import mans_b200 as mb
    from mans_b200.batch import Batch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    count = args.items or 4096
    items, total = mixed_layout(count)
    U = sum(it["bytes"] for it in items)
    pool = gen_mixed_device(items, total, seed=3 + rank)
    tdt = {2: torch.uint16, 4: torch.uint32}
    xs = [pool[it["off"]:it["off"] + it["bytes"]].view(tdt[it["elem"]]) for it in items]
    codes = [mb.MANS_U16 if it["elem"] == 2 else mb.MANS_U32 for it in items]
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    lib = mb.load()
    p = args.precision

    # ---- plain path: one workspace, one call per buffer, back to back on one stream
    ws = mb.Workspace(max(it["bytes"] for it in items))
    scap = max(mb.max_compressed_size(c, it["n"]) for c, it in zip(codes, items))
    scratch = torch.empty(scap, dtype=torch.uint8, device="cuda")
    sizes0 = torch.zeros(count, dtype=torch.int64, device="cuda")
    for i, it in enumerate(items):  # stream sizes, to lay out the output pools
        r = lib.mans_compress(ws.h, codes[i], xs[i].data_ptr(), it["n"], scratch.data_ptr(), scap,
                              sizes0.data_ptr() + 8 * i, p, sh)
        if r:
            raise mb.MansError(r, "mans_compress")
    ws.check(stream, "sizes")
    csz = sizes0.tolist()
    del scratch
    ooff, o = [], 0
    for c in csz:
        ooff.append(o)
        o += (c + 255) // 256 * 256
    out_total = o
    outA = torch.zeros(out_total, dtype=torch.uint8, device="cuda")
    outB = torch.zeros(out_total, dtype=torch.uint8, device="cuda")
    dec = torch.zeros(total, dtype=torch.uint8, device="cuda")
    sizesA = torch.zeros(count, dtype=torch.int64, device="cuda")
    sizesB = torch.zeros(count, dtype=torch.int64, device="cuda")
    caps = [(c + 255) // 256 * 256 for c in csz]
    pa, pb, pd = outA.data_ptr(), outB.data_ptr(), dec.data_ptr()
    c_args = [(ws.h, codes[i], xs[i].data_ptr(), it["n"], pa + ooff[i], caps[i],
               sizesA.data_ptr() + 8 * i, p, sh) for i, it in enumerate(items)]
    d_args = [(ws.h, codes[i], pa + ooff[i], csz[i], pd + it["off"], it["n"], sh)
              for i, it in enumerate(items)]
    f_c, f_d = lib.mans_compress, lib.mans_decompress

    def plain_compress():
        for a in c_args:
            if f_c(*a):
                raise RuntimeError("mans_compress failed")

    def plain_decompress():
        for a in d_args:
            if f_d(*a):
                raise RuntimeError("mans_decompress failed")

    def timed(fns, steps):
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(len(fns) + 1)] for _ in range(steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(steps):
            evs[k][0].record(stream)
            for j, f in enumerate(fns):
                f()
                evs[k][j + 1].record(stream)
        torch.cuda.synchronize()
        return [sum(evs[k][j].elapsed_time(evs[k][j + 1]) for k in range(steps)) / steps
                for j in range(len(fns))]

    for _ in range(max(3, args.warmup)):
        plain_compress()
        plain_decompress()
    ws.check(stream, "plain warm-up")
    plain_ok = bool(torch.equal(dec, pool)) and sizesA.tolist() == csz
    with ClockSampler(local) as clk_plain:
        plain_c, plain_d = timed([plain_compress, plain_decompress], args.steps)
    ws.check(stream, "plain timed")

    # plain calls replayed from CUDA graphs (launch cost removed), for reference
    s2 = torch.cuda.Stream()
    s2.wait_stream(stream)
    gpc, gpd = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(gpc, stream=s2):
        for a in c_args:
            f_c(*(a[:-1] + (s2.cuda_stream,)))
    with torch.cuda.graph(gpd, stream=s2):
        for a in d_args:
            f_d(*(a[:-1] + (s2.cuda_stream,)))
    for _ in range(2):
        gpc.replay()
        gpd.replay()
    pg_c, pg_d = timed([gpc.replay, gpd.replay], args.steps)
    ws.check(stream, "plain graph")
    plain_ok = plain_ok and bool(torch.equal(dec, pool))
    del gpc, gpd

    # ---- batched path: one call per direction, captured in a CUDA graph
    batch = Batch(count, U, args.merged_ratio)
    outsB = [outB[ooff[i]:ooff[i] + caps[i]] for i in range(count)]
    decs = [dec[it["off"]:it["off"] + it["bytes"]].view(tdt[it["elem"]]) for it in items]
    items_c = Batch.compress_items(xs, outsB, sizesB, p)
    items_d = Batch.decompress_items(outsB, csz, decs)
    dec.zero_()
    batch.compress_async(items_c)
    batch.check(count, stream, "batch compress")
    batch.decompress_async(items_d)
    batch.check(count, stream, "batch decompress")
    stream_equal = bool(torch.equal(outA, outB)) and sizesB.tolist() == csz
    batch_ok = bool(torch.equal(dec, pool))
    tuned_ms = batch.autotune(items_c, stream) if not args.no_autotune else None
    sched, sched_max = batch.schedule()
    sched_full, _ = batch.schedule_ex()
    batch.set_timing(True)
    for _ in range(3):
        batch.compress_async(items_c)
        batch.decompress_async(items_d)
    st = batch.stage_times()
    batch.set_timing(False)
    n_rec = max(1, st["compress_calls"])
    stage_ms = {k: st[k] / n_rec for k in ("map", "plan", "encode", "decode_plan", "decode", "unmap")}
    gbc, gbd = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    s2.wait_stream(stream)
    with torch.cuda.graph(gbc, stream=s2):
        batch.compress_async(items_c, s2)
    with torch.cuda.graph(gbd, stream=s2):
        batch.decompress_async(items_d, s2)
    for _ in range(max(3, args.warmup)):
        gbc.replay()
        gbd.replay()
    dec.zero_()
    outB.zero_()
    with ClockSampler(local) as clk:
        b_c, b_d = timed([gbc.replay, gbd.replay], args.steps)
    batch.check(count, stream, "batch timed")
    stream_equal = stream_equal and bool(torch.equal(outA, outB))
    batch_ok = batch_ok and bool(torch.equal(dec, pool))

    b_c, b_d, plain_c, plain_d, pg_c, pg_d = reduce_max_over_ranks(
        [b_c, b_d, plain_c, plain_d, pg_c, pg_d], dist)
    gbs = lambda ms: round(world * U / (ms / 1e3) / 1e9, 3)  # noqa: E731

    # ---- end to end through the public API with host buffers: every buffer
    # is uploaded, compressed, its stream downloaded and uploaded again,
    # decompressed and downloaded. The buffers are cut into chunks of about
    # equal bytes that alternate between two streams, each with its own batch
    # handle, so one chunk's downloads overlap the next chunk's uploads (PCIe
    # is full duplex); only each stream's own bytes cross the bus.
    e2e = None
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 0
    need = total + out_total + total
    if avail > 2 * need and not getattr(args, "no_e2e", False):
        del gbc, gbd
        batch.close()
        n_chunks = 8
        chunks, lo, acc = [], 0, 0
        for i, it in enumerate(items):
            acc += it["bytes"]
            if acc >= U / n_chunks * (len(chunks) + 1) or i == count - 1:
                chunks.append((lo, i + 1))
                lo = i + 1
        cb = max(sum(items[j]["bytes"] for j in range(a_, b_)) for a_, b_ in chunks)
        ci = max(b_ - a_ for a_, b_ in chunks)
        pair = [Batch(ci, cb, args.merged_ratio), Batch(ci, cb, args.merged_ratio)]
        for bh in pair:
            bh.set_schedule_ex(sched_full)
        streams_e = [torch.cuda.Stream(), torch.cuda.Stream()]
        work = []
        for k, (a_, b_) in enumerate(chunks):
            i0, i1 = items[a_]["off"], items[b_ - 1]["off"] + items[b_ - 1]["bytes"]
            o0, o1 = ooff[a_], ooff[b_ - 1] + caps[b_ - 1]
            work.append({"k": k, "a": a_, "b": b_, "i": (i0, i1), "o": (o0, o1),
                         "ic": Batch.compress_items(xs[a_:b_], outsB[a_:b_], sizesB[a_:b_], p),
                         "id": Batch.decompress_items(outsB[a_:b_], csz[a_:b_], decs[a_:b_])})
        h_in = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        h_in.copy_(pool)
        h_s = torch.empty(out_total, dtype=torch.uint8, pin_memory=True)
        h_sz = torch.empty(count, dtype=torch.int64, pin_memory=True)
        h_out = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        pool.zero_()
        outB.zero_()
        dec.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for se in streams_e:
            se.wait_stream(stream)
        for w in work:
            se, bh = streams_e[w["k"] % 2], pair[w["k"] % 2]
            (i0, i1), (o0, o1), a_, b_ = w["i"], w["o"], w["a"], w["b"]
            with torch.cuda.stream(se):
                pool[i0:i1].copy_(h_in[i0:i1], non_blocking=True)
                bh.compress_async(w["ic"], se)
                h_sz[a_:b_].copy_(sizesB[a_:b_], non_blocking=True)
                h_s[o0:o1].copy_(outB[o0:o1], non_blocking=True)
                outB[o0:o1].copy_(h_s[o0:o1], non_blocking=True)
                bh.decompress_async(w["id"], se)
                h_out[i0:i1].copy_(dec[i0:i1], non_blocking=True)
        for se in streams_e:
            stream.wait_stream(se)
        b.record(stream)
        torch.cuda.synchronize()
        for w in work:
            pair[w["k"] % 2].check(w["b"] - w["a"], streams_e[w["k"] % 2], "e2e")
        e2e_ms = a.elapsed_time(b)
        e2e = {"value": gbs(e2e_ms), "unit": "GB/s", "h2d_bytes_per_step": total + out_total,
               "d2h_bytes_per_step": 8 * count + out_total + total, "ms_per_step": round(e2e_ms, 2),
               "mode": f"{len(chunks)} chunks of buffers pipelined over 2 streams",
               "bit_exact": bool(torch.equal(h_out, h_in)) and h_sz.tolist() == csz}
        for bh in pair:
            bh.close()
        del h_in, h_s, h_out
        batch = None

    result = None
    if rank == 0:
        peak, peak_src = hbm_peak()
        hdr_n = outA.view(torch.int32)[torch.tensor([(x + 8) // 4 for x in ooff], device="cuda")]
        M = int(hdr_n.to(torch.int64).sum().item())
        C_ = sum(csz)
        algo = {"map": U + M, "plan": 0, "encode": M + C_, "decode_plan": 0, "decode": C_ + M,
                "unmap": M + U}
        names = {"map": "batch_map_kernel", "encode": "batch_encode_kernel",
                 "decode": "batch_decode_kernel", "unmap": "batch_unmap_kernel"}
        dom = max(names, key=lambda k: stage_ms[k])
        achieved = algo[dom] / (stage_ms[dom] / 1e3) / 1e9
        result = {
            "metric": METRIC, "value": gbs(b_c + b_d), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(b_c + b_d, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16+u32",
            "data": "synthetic",
            "config": {"workload": MIXED_DESC.format(count=count)
                       + "; per step every buffer is compressed and decompressed once",
                       "buffers": count, "uncompressed_bytes": U, "precision": p,
                       "merged_ratio_pct": args.merged_ratio or 210,
                       "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "batched": {"compress_gbs": gbs(b_c), "decompress_gbs": gbs(b_d),
                        "round_trip_gbs": gbs(b_c + b_d), "ms_compress": round(b_c, 3),
                        "ms_decompress": round(b_d, 3), "graph": True,
                        "schedule_ctas_per_sm": sched, "schedule_max": sched_max,
                        "schedule": sched_full,
                        "autotune_best_ms": tuned_ms,
                        "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()}},
            "plain": {"compress_gbs": gbs(plain_c), "decompress_gbs": gbs(plain_d),
                      "round_trip_gbs": gbs(plain_c + plain_d), "ms_compress": round(plain_c, 3),
                      "ms_decompress": round(plain_d, 3),
                      "calls": "one mans_compress / mans_decompress per buffer, back to back"},
            "plain_graph": {"round_trip_gbs": gbs(pg_c + pg_d), "ms_compress": round(pg_c, 3),
                            "ms_decompress": round(pg_d, 3)},
            "batched_vs_plain": round((plain_c + plain_d) / (b_c + b_d), 3),
            "batched_vs_plain_graph": round((pg_c + pg_d) / (b_c + b_d), 3),
            "compressed_bytes": C_, "mapped_bytes": M, "compression_ratio": round(U / C_, 4),
            "bit_exact_round_trip": plain_ok and batch_ok,
            "batched_streams_equal_plain": stream_equal,
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": round(achieved, 1),
                         "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None},
            "e2e": e2e,
            "gpu_launches": 8 * args.steps,
            "clocks": clk.summary(), "clocks_plain": clk_plain.summary(),
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if batch is not None:
        batch.close()
    ws.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = mixed_cpu_sample(reps=3, warm=1)
    return result


# ---------------------------------------------------------------- serving
SERVE_DESC = ("serve_c5: {R} requests, Poisson arrivals at {rate:g} GB/s offered, sizes log-uniform "
              "in [16 KiB, 256 MiB] (a seeded corpus of {D} buffers, alternating uint16 gradients and "
              "uint32 Laplace codes as in mixed_c3), 50/50 compress/decompress, decompress inputs are "
              "earlier compress outputs of the same buffers; 64 GiB HBM budget; seed 5")


def serve_trace(srv, reqs, arrivals_s, corpus, streams, check: bool):
    """Submit reqs at their arrival times (a submitter thread) and collect,
    check and release every completion. Returns per-request records."""
    import torch

    from mans_b200 import serve
    R = len(reqs)
    t0 = serve.clock_ns() + 50_000_000
    err = []

    def submitter():
        try:
            for k, (op, i) in enumerate(reqs):
                target = t0 + int(arrivals_s[k] * 1e9)
                now = serve.clock_ns()
                if target > now + 200_000:
                    time.sleep((target - now) / 1e9)
                x, code, n = corpus[i]
                if op == 0:
                    srv.submit(serve.COMPRESS, code, n, x.data_ptr(), precision=10, tag=k,
                               arrival_ns=target)
                else:
                    s = streams[i]
                    srv.submit(serve.DECOMPRESS, code, n, s.data_ptr(), in_bytes=s.numel(), tag=k,
                               arrival_ns=target)
        except Exception as e:  # pragma: no cover - reported below
            err.append(e)

    # The check must not allocate: a large allocation that misses torch's
    # cache calls cudaMalloc / cudaFree, which synchronise the device and
    # stall the server's scheduler thread along with it.
    cmp = torch.empty(max(max(int(s.numel()) for s in streams),
                          max(int(c[0].numel() * c[0].element_size()) for c in corpus)),
                      dtype=torch.bool, device="cuda") if check else None

    def same(a, b) -> bool:
        torch.eq(a, b, out=cmp[:a.numel()])
        return bool(cmp[:a.numel()].all())

    th = threading.Thread(target=submitter, daemon=True)
    th.start()
    rec = np.zeros((R, 5), dtype=np.float64)  # latency ns, queued ns, batch items, ok, done time ns
    n = 0
    bad = 0
    while n < R:
        if err:
            raise err[0]
        for c in srv.poll(timeout_us=5000):
            k = c.tag
            op, i = reqs[k]
            ok = c.status == 0
            if ok and check:
                if op == 0:
                    ref = streams[i]
                    ok = c.out_bytes == ref.numel() and same(serve.view_device(c.d_out, c.out_bytes), ref)
                else:
                    x = corpus[i][0].view(torch.uint8)
                    ok = c.out_bytes == x.numel() and same(serve.view_device(c.d_out, c.out_bytes), x)
            if c.status == 0:
                srv.release(c.ticket)
            bad += 0 if ok else 1
            rec[k] = (c.latency_ns, c.queued_ns, c.batch_items, 1.0 if ok else 0.0, serve.clock_ns() - t0)
            n += 1
    th.join()
    return rec, bad


def serve_summary(rec, reqs, sizes_b, arrivals_s):
    lat = rec[:, 0] / 1e6
    ops = np.array([op for op, _ in reqs])
    nbytes = np.array([sizes_b[i] for _, i in reqs], dtype=np.float64)
    span = rec[:, 4].max() / 1e9  # last completion, from the trace's time origin
    first = float(arrivals_s[0])
    out = {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
           "mean_ms": round(float(lat.mean()), 3),
           "compress_p50_ms": round(float(np.percentile(lat[ops == 0], 50)), 3) if (ops == 0).any() else None,
           "compress_p99_ms": round(float(np.percentile(lat[ops == 0], 99)), 3) if (ops == 0).any() else None,
           "decompress_p50_ms": round(float(np.percentile(lat[ops == 1], 50)), 3) if (ops == 1).any() else None,
           "decompress_p99_ms": round(float(np.percentile(lat[ops == 1], 99)), 3) if (ops == 1).any() else None,
           "queued_p50_ms": round(float(np.percentile(rec[:, 1] / 1e6, 50)), 3),
           "mean_batch_items": round(float(rec[:, 2].mean()), 2),
           "aggregate_gbs": round(float(nbytes.sum() / max(span - first, 1e-9) / 1e9), 3),
           "requests": len(reqs), "bytes": int(nbytes.sum()), "all_identical": bool(rec[:, 3].all())}
    return out


def run_serve(args):
    import torch

    import mans_b200 as mb
    from mans_b200 import serve

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    R = args.requests or 100_000
    D = args.corpus or 256
    rate = args.rate
    rng = np.random.default_rng(5)
    sz = np.exp(rng.uniform(np.log(16 << 10), np.log(256 << 20), D))
    sz = (np.floor(sz / 1024) * 1024).astype(np.int64)
    ab = rng.uniform(-1000, 1000, (D, 2))
    items, off = [], 0
    for i, nb in enumerate(sz.tolist()):
        elem = 2 if i % 2 == 0 else 4
        items.append({"elem": elem, "n": nb // elem, "bytes": nb // elem * elem, "off": off,
                      "a": float(ab[i, 0]), "b": float(ab[i, 1])})
        off += (nb + 255) // 256 * 256
    pool = gen_mixed_device(items, off, seed=5 + rank)
    tdt = {2: torch.uint16, 4: torch.uint32}
    corpus = [(pool[it["off"]:it["off"] + it["bytes"]].view(tdt[it["elem"]]),
               mb.MANS_U16 if it["elem"] == 2 else mb.MANS_U32, it["n"]) for it in items]
    sizes_b = [it["bytes"] for it in items]
    # compressed corpus through the single-buffer path (the reference result of every request)
    ws = mb.Workspace(max(sizes_b))
    streams = [mb.compress(x, 10, ws=ws) for x, _, _ in corpus]
    ws.close()
    ops = (rng.random(R) < 0.5).astype(np.int64)
    idx = rng.integers(0, D, R)
    reqs = [(int(o), int(i)) for o, i in zip(ops, idx)]
    mean_b = float(np.mean([sizes_b[i] for i in idx]))
    lam = rate * 1e9 / mean_b
    arrivals = np.cumsum(rng.exponential(1.0 / lam, R))
    budget = 64 << 30
    results = {}
    R_sat = min(R, args.saturation_requests)
    for name, kw in (("batched", dict(max_batch_bytes=1 << 30, max_batch_items=1024, lanes=2,
                                      merged_ratio_pct=args.merged_ratio)),
                     ("plain", dict(max_batch_bytes=max(sizes_b), plain=True))):
        srv = serve.Server(budget, **kw)
        dev_bytes = srv.stats()["device_bytes"]
        clk = ClockSampler(local)
        with clk:
            rec, bad = serve_trace(srv, reqs, arrivals, corpus, streams, check=not args.no_check)
        st = srv.stats()
        summ = serve_summary(rec, reqs, sizes_b, arrivals)
        summ.update({"launches": st["launches"], "arena_peak_bytes": st["arena_peak"],
                     "device_bytes": dev_bytes, "mismatches": bad, "clocks": clk.summary()})
        # saturation: every request of a prefix queued at once
        rec2, bad2 = serve_trace(srv, reqs[:R_sat], np.zeros(R_sat), corpus, streams, check=False)
        s2 = serve_summary(rec2, reqs[:R_sat], sizes_b, np.zeros(R_sat))
        summ["saturated"] = {"requests": R_sat, "aggregate_gbs": s2["aggregate_gbs"],
                             "p50_ms": s2["p50_ms"], "p99_ms": s2["p99_ms"],
                             "mean_batch_items": s2["mean_batch_items"], "errors": bad2}
        srv.close()
        results[name] = summ
    b, p = results["batched"], results["plain"]
    line = {
        "metric": METRIC, "value": b["aggregate_gbs"], "unit": "GB/s", "n_gpus": world,
        "steps": 1, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16+u32", "data": "synthetic",
        "config": {"workload": SERVE_DESC.format(R=R, rate=rate, D=D), "offered_gbs": rate,
                   "arrival_rate_per_s": round(lam, 1), "hbm_budget_bytes": budget,
                   "parallelism": "single GPU"},
        "p50_ms": b["p50_ms"], "p99_ms": b["p99_ms"],
        "batched": b, "plain": p,
        "p99_plain_over_batched": round(p["p99_ms"] / b["p99_ms"], 3) if b["p99_ms"] else None,
        "saturated_batched_vs_plain": round(b["saturated"]["aggregate_gbs"] / p["saturated"]["aggregate_gbs"], 3),
        "bit_exact": b["all_identical"] and p["all_identical"],
        "e2e": None, "e2e_note": "requests reference device-resident buffers; see mixed_c3 / default runs for host-buffer e2e",
        "gpu_launches": None,
    }
    if rank == 0:
        return line
    return None


def check_oracle(args, x, s) -> bool:
    """The device stream s of input x equals the oracle's, byte for byte."""
    from oracle import pyoracle as O
    from tests.helpers import to_host
    xh = to_host(x, np.uint32 if x.element_size() == 4 else np.uint16)
    want = O.compress_par(xh, args.precision)
    got = to_host(s)
    return bool(got.size == want.size and np.array_equal(got, want))


def _parse_floats(text: str, keys: dict) -> dict:
    out = {}
    for name, label in keys.items():
        for line in text.splitlines():
            if label in line:
                try:
                    out[name] = float(line.split(label, 1)[1].strip().split()[0])
                except (ValueError, IndexError):
                    pass
    return out


def _ours_per_stage(x, reps: int = 10) -> dict:
    """Per-kernel milliseconds of this library on device tensor x (events
    the library records around each launch), after warm-up."""
    import torch

    import mans_b200 as mb
    n = x.numel()
    ws = mb.Workspace(n * x.element_size())
    cap = mb.max_compressed_size(mb.dtype_code(x), n)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    back = torch.empty_like(x)
    for _ in range(3):
        mb.compress_into(ws, x, out, size, 10)
        mb.decompress_into(ws, out, cap, back)
    ws.check(None, "warm-up")
    ws.set_timing(True)
    for _ in range(reps):
        mb.compress_into(ws, x, out, size, 10)
        mb.decompress_into(ws, out, cap, back)
    kt = ws.kernel_times()
    ws.set_timing(False)
    ws.check(None, "timed")
    ok = bool(torch.equal(back.view(torch.uint8), x.view(torch.uint8)))
    ws.close()
    c, d = max(1, kt["compress_calls"]), max(1, kt["decompress_calls"])
    r = {"map_ms": kt["map"] / c, "encode_ms": kt["encode"] / c, "decode_ms": kt["decode"] / d,
         "unmap_ms": kt["unmap"] / d, "round_trip_ok": ok}
    return {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()}


def reference_gpu(args) -> dict:
    """The reference's own GPU path, built from its sources under oracle/_ref
    (oracle/Makefile), timed on this GPU on the same inputs as this library:
    the V15 uint16 mapper (mapping/nv/mappingV15_fused_uint16.cu, its own
    CUDA-event timing, :856-869 and :971-985) and the V9 uint32 mapper
    (mapping/nv/mappingV9_fuse.cu:841-919) each followed by the include/ans
    codec (ansEncode / ansDecode, timed by oracle/ref_ans_driver in its
    "time" mode: CUDA events and a host clock per call as
    examples/compress.cu:45-63). Inputs the reference handles: config 1
    (4,194,304 uint16) and a 2^27-element slice of the uint32 detector
    frames (the reference's uint32 mapper sizes its scratch with an int and
    fails at 2^28 elements, mappingV9_fuse.cu:803). Lazy module loading is
    off (CUDA_MODULE_LOADING=EAGER) so that no kernel's first launch pays for
    loading code."""
    import subprocess
    import tempfile

    import torch

    from mans_b200 import workloads as W
    ref = os.path.join(ROOT, "oracle", "_ref")
    bins = {k: os.path.join(ref, k) for k in ("mappingV15", "mappingV9", "ref_ans_driver")}
    missing = [k for k, v in bins.items() if not os.path.exists(v)]
    if missing:
        return {"unavailable": f"reference binaries not built: {', '.join(missing)}"}
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    res = {"what": "per-stage milliseconds of the reference's GPU code and of this library on "
                   "the same inputs, same GPU, same run"}

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{os.path.basename(cmd[0])} rc={r.returncode}: {r.stderr[-300:]}")
        return r.stdout

    with tempfile.TemporaryDirectory() as td:
        cases = [("laplace_u16_c1", W.laplace_u16(W.C1_N, 1), "mappingV15"),
                 ("detector_u32_2p27", W.detector_u32(1 << 27, 2), "mappingV9")]
        for name, x, mapper in cases:
            fi, fm = os.path.join(td, name + ".bin"), os.path.join(td, name + ".adm")
            x.tofile(fi)
            rec = {"elements": int(x.size), "bytes": int(x.nbytes)}
            if mapper == "mappingV15":
                txt = run([bins[mapper], fi, fm])
                rec["reference"] = _parse_floats(txt, {
                    "map_ms": "Total Cmp Time:", "map_adm_kernel_ms": "ADM cost",
                    "map_prefix_sum_ms": "Prefix-sum cost", "map_concat_ms": "Concat cost",
                    "unmap_ms": "Total cost"})
            else:
                txt = run([bins[mapper], fi, fm, "uint32"])
                rec["reference"] = _parse_floats(txt, {"map_ms": "Compression cost",
                                                       "unmap_ms": "Decompression cost"})
            rec["reference"]["mapped_bytes"] = os.path.getsize(fm)
            txt = run([bins["ref_ans_driver"], "time", "10", fm, "5"])
            line = next((l for l in txt.splitlines() if l.startswith("REFTIME")), "")
            kv = dict(t.split("=", 1) for t in line.split()[1:] if "=" in t)
            rec["reference"].update({
                "encode_ms": float(kv.get("encode_event_ms", "nan")),
                "encode_wall_ms": float(kv.get("encode_wall_ms", "nan")),
                "decode_ms": float(kv.get("decode_event_ms", "nan")),
                "decode_wall_ms": float(kv.get("decode_wall_ms", "nan")),
                "rans_round_trip_ok": kv.get("roundtrip") == "ok"})
            rec["reference"]["pipeline_ms"] = round(sum(
                rec["reference"].get(k, 0.0) for k in ("map_ms", "encode_ms", "decode_ms", "unmap_ms")), 4)
            d = torch.from_numpy(x.view(np.uint8).copy()).cuda().view(
                torch.uint16 if x.dtype == np.uint16 else torch.uint32)
            rec["mans"] = _ours_per_stage(d)
            rec["mans"]["pipeline_ms"] = round(sum(
                rec["mans"][k] for k in ("map_ms", "encode_ms", "decode_ms", "unmap_ms")), 4)
            rec["speedup"] = round(rec["reference"]["pipeline_ms"] / rec["mans"]["pipeline_ms"], 2) \
                if rec["mans"]["pipeline_ms"] else None
            res[name] = rec
            del d
    return res


def sub_records(args) -> dict:
    """The batched (config 3) and served (config 5) forms and the reference's
    own GPU path, measured after the single-buffer headline in the same run
    (one GPU): the metric's "batched vs plain" and "p50/p99 latency" parts."""
    import copy

    import torch
    out = {}
    sub = copy.copy(args)
    torch.cuda.empty_cache()  # the headline's buffers, cached by torch
    sub.no_cpu_baseline = True
    t0 = time.time()
    try:
        sub.items, sub.steps, sub.warmup, sub.no_e2e = 0, args.sub_steps, 3, True
        out["mixed_c3"] = run_mixed(sub)
        out["mixed_c3"]["seconds"] = round(time.time() - t0, 1)
    except Exception as e:  # reported, never hidden
        out["mixed_c3"] = {"error": f"{type(e).__name__}: {e}"}
    torch.cuda.empty_cache()  # the serving loop reserves its whole HBM budget up front
    t0 = time.time()
    try:
        sub.requests, sub.steps = args.sub_requests, 1
        out["serve_c5"] = run_serve(sub)
        out["serve_c5"]["seconds"] = round(time.time() - t0, 1)
    except Exception as e:
        out["serve_c5"] = {"error": f"{type(e).__name__}: {e}"}
    torch.cuda.empty_cache()
    t0 = time.time()
    try:
        out["reference_gpu"] = reference_gpu(args)
        out["reference_gpu"]["seconds"] = round(time.time() - t0, 1)
    except Exception as e:
        out["reference_gpu"] = {"error": f"{type(e).__name__}: {e}"}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "mixed_c3":
        line = run_mixed(args)
    elif args.workload == "serve_c5":
        line = run_serve(args)
    else:
        line = run_mans(args)
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if line is not None and world == 1 and args.workload == "detector_u32" and not args.n \
                and not args.no_sub:
            line.update(sub_records(args))
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
