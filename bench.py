"""Benchmark of the B200 fmm2d evaluation path.

Workload (default): Laplace ``lfmm2d_st_cd_g`` on 10^7 sources + 10^7
targets uniform in [0,1]^2, complex charges and dipole strengths N(0,1),
unit dipole vectors at angle U[0, 2pi), eps = 1e-6 in the mixed-precision
form -- seeded synthetic inputs of the shapes the reference's Laplace FMM
is quoted on.  ``fp64_plain``: the same inputs in the plain form, all-FP64
at eps = 1e-12 (``--plain-eps``).

One step = one full evaluation (tree, lists, all FMM passes, near field,
outputs in input order) through the library's C ABI.
  value  : points/s with inputs and outputs resident in HBM (the C ABI is
           called with device pointers).
  e2e    : points/s through the same C-ABI call with pinned HOST buffers;
           host->device and device->host copies are inside the call.
Timing: CUDA events on the stream the library runs on (set with
fmm2d_b200_set_stream), W untimed warm-up steps, K timed steps bracketed
by a barrier and cuda synchronize; inputs (0.8 GB) exceed the 126 MB L2.

``--impl reference`` times the reference's own C translation (compiled
from the reference sources into oracle/_ref/ by oracle/Makefile) on the
host cores: each step runs one bounded sample of the same workload per
host thread, concurrently.

Multi-GPU (``torchrun --nproc-per-node N``): independent replicas, one
full problem per GPU (the evaluation path does not shard), value = all
points of all ranks / max step time over ranks.

Serving (``serving`` key, rank 0): the stream of the serving configuration
-- requests with N log-uniform in [1e3, 1e6] points, uniform or Gaussian
blobs (sigma 0.01) in [0,1]^2, 70 % Laplace lfmm2d_s_c_g at eps in
{1e-3, 1e-6, 1e-9}, 30 % Helmholtz hfmm2d_s_c_g with zk ~ U[1, 50] at eps
1e-6, complex charges N(0,1) -- through the library's request loop
(fmm2d_b200_server_*) with an HBM budget of 120 GB.  Arrivals are Poisson
at 70 % of the throughput measured on a saturating burst of the same
stream; latency = submission to completion (host arrays, copies
included); p50 / p99 over all requests.  Beside it, the same requests one
at a time in all-FP64 mode (one slot).  ``--serve-requests`` sets the
stream length (20,000 by default, as the configuration names); the
one-at-a-time baseline runs the first --serve-baseline requests of it.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "points/s Laplace FMM eps 1e-6 mixed vs FP64 plain, 1 B200; serving p50/p99 ms"
P = ctypes.c_void_p
NS_DEFAULT = 10_000_000
NT_DEFAULT = 10_000_000


def make_inputs(ns, nt, seed):
    rng = np.random.default_rng(seed)
    src = rng.random((ns, 2))
    trg = rng.random((nt, 2))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0.0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)], axis=1)
    return src, trg, q, d, v


# DRAM bytes (read + write) per launch of the dominant kernel at 2e6 + 2e6
# uniform points, from `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum`
# on the bench command with --ns 2000000 --nt 2000000 (the summary with the
# full command is kept in profiles/)
TRAFFIC_2E6 = {
    ("mixed", "m2l"): (249.3e6, "profiles/kernels_mixed_2e6_dram.md: m2l_win_kernel<2,20,4> "
                                "103.9 MB read + 145.4 MB write at 2e6+2e6, scaled by points"),
    ("mixed", "p2p"): (661.8e6, "profiles/kernels_mixed_2e6_dram.md: p2p_flat_kernel "
                                "447.6 MB read + 214.2 MB write at 2e6+2e6, scaled by points"),
}


def read_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region.

    The sampler is started and its first sample awaited before the timed
    region begins; the samples kept are those from mark() on, plus the first
    one after stop() is called (short timed regions fall between samples)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.lock = threading.Lock()
        self.first = threading.Event()
        self.mark_at = 0
        self.reader = None

    def _read(self):
        for line in self.proc.stdout:
            with self.lock:
                self.lines.append(line)
            self.first.set()

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        self.first.wait(10.0)

    def mark(self):
        with self.lock:
            self.mark_at = len(self.lines)

    def stop(self):
        if self.proc is None:
            return None
        with self.lock:
            n_end = len(self.lines)
        t0 = time.time()
        while time.time() - t0 < 2.0:
            with self.lock:
                if len(self.lines) > n_end:
                    break
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        self.reader.join(5.0)  # ends at the pipe's end of file
        with self.lock:
            out = "".join(self.lines[self.mark_at:n_end + 1])
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def parse_profile(s):
    out = {}
    for kv in s.split(";"):
        if "=" in kv:
            k, v = kv.split("=", 1)
            out[k] = float(v)
    return out


def max_over_ranks(value, ws, device=None):
    """The largest of a per-rank value over all ranks (the step time of the
    rank that finished last); the value itself on one rank."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(points_per_rank, ws, step_ms):
    """points/s of the whole job: every rank's points over the slowest
    rank's step time (replicas: each rank evaluates a full problem)."""
    return ws * points_per_rank / (step_ms * 1e-3)


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    """The reference's C translation on the host cores."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import refimpl
    if not refimpl.have_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libfmm2d_ref.so not built (reference sources absent at build time)"}))
        return 0
    R = refimpl.ref()
    threads = args.cpu_threads or (os.cpu_count() or 1)
    ns, nt = args.cpu_sample, args.cpu_sample
    inputs = [make_inputs(ns, nt, 1000 + t) for t in range(threads)]
    eps = ctypes.c_double(args.eps)

    def one(t):
        src, trg, q, d, v = inputs[t]
        pot = np.zeros(ns, complex)
        grad = np.zeros((ns, 2), complex)
        pt = np.zeros(nt, complex)
        gt = np.zeros((nt, 2), complex)
        ier = ctypes.c_int(0)
        R.lfmm2d_st_cd_g_(ctypes.byref(eps), ctypes.byref(ctypes.c_int(ns)),
                          src.ctypes.data_as(P), q.ctypes.data_as(P),
                          d.ctypes.data_as(P), v.ctypes.data_as(P),
                          pot.ctypes.data_as(P), grad.ctypes.data_as(P),
                          ctypes.byref(ctypes.c_int(nt)), trg.ctypes.data_as(P),
                          pt.ctypes.data_as(P), gt.ctypes.data_as(P),
                          ctypes.byref(ier))

    def step():
        ths = [threading.Thread(target=one, args=(t,)) for t in range(threads)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(args.steps)]
    tm = sum(times) / len(times)
    value = threads * (ns + nt) / tm
    full = None
    if args.reference_full:
        # one call of the full workload (sequential: the C translation has no
        # threads), timed once; minutes of host time, hence off by default
        src, trg, q, d, v = make_inputs(args.ns, args.nt, 7)
        outs = [np.zeros(args.ns, complex), np.zeros((args.ns, 2), complex),
                np.zeros(args.nt, complex), np.zeros((args.nt, 2), complex)]
        ierf = ctypes.c_int(0)
        t0 = time.perf_counter()
        R.lfmm2d_st_cd_g_(ctypes.byref(eps), ctypes.byref(ctypes.c_int(args.ns)),
                          src.ctypes.data_as(P), q.ctypes.data_as(P), d.ctypes.data_as(P),
                          v.ctypes.data_as(P), outs[0].ctypes.data_as(P), outs[1].ctypes.data_as(P),
                          ctypes.byref(ctypes.c_int(args.nt)), trg.ctypes.data_as(P),
                          outs[2].ctypes.data_as(P), outs[3].ctypes.data_as(P), ctypes.byref(ierf))
        tf = time.perf_counter() - t0
        full = {"seconds": tf, "points_s": (args.ns + args.nt) / tf, "cores": 1, "ier": ierf.value,
                "call": f"lfmm2d_st_cd_g_ {args.ns}+{args.nt} points eps={args.eps:g}, one call"}
    sample = (f"{threads} concurrent lfmm2d_st_cd_g calls of {ns}+{nt} points "
              f"(same distributions, eps={args.eps:g}) per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tm * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "lfmm2d_st_cd_g uniform 1e7+1e7 eps 1e-6 (bounded CPU sample)",
                   "precision": "fp64", "sample": sample},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads,
                         "kind": "reference", "sample": sample, "full_size_once": full,
                         "openmp_fortran": openmp_fortran_probe()},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def cpu_baseline_sample(args):
    """A bounded run of the reference C translation (1 core per call, all
    host threads concurrently) for the cpu_baseline field."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import refimpl
    if not refimpl.have_ref():
        return None
    R = refimpl.ref()
    threads = args.cpu_threads or (os.cpu_count() or 1)
    ns = nt = args.cpu_sample
    inputs = [make_inputs(ns, nt, 2000 + t) for t in range(threads)]
    eps = ctypes.c_double(args.eps)

    def one(t):
        src, trg, q, d, v = inputs[t]
        outs = [np.zeros(ns, complex), np.zeros((ns, 2), complex),
                np.zeros(nt, complex), np.zeros((nt, 2), complex)]
        ier = ctypes.c_int(0)
        R.lfmm2d_st_cd_g_(ctypes.byref(eps), ctypes.byref(ctypes.c_int(ns)),
                          src.ctypes.data_as(P), q.ctypes.data_as(P),
                          d.ctypes.data_as(P), v.ctypes.data_as(P),
                          outs[0].ctypes.data_as(P), outs[1].ctypes.data_as(P),
                          ctypes.byref(ctypes.c_int(nt)), trg.ctypes.data_as(P),
                          outs[2].ctypes.data_as(P), outs[3].ctypes.data_as(P),
                          ctypes.byref(ier))

    ths = [threading.Thread(target=one, args=(t,)) for t in range(threads)]
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    dt = time.perf_counter() - t0
    sample = (f"{threads} concurrent reference lfmm2d_st_cd_g calls of "
              f"{ns}+{nt} points, eps={args.eps:g}, {dt:.1f} s wall")
    return {"value": threads * (ns + nt) / dt, "unit": "points/s",
            "cores": threads, "kind": "reference", "sample": sample,
            "openmp_fortran": openmp_fortran_probe()}


def openmp_fortran_probe():
    """The reference's preferred CPU baseline is its OpenMP Fortran library,
    which needs gfortran on the host: report whether this host has one."""
    import shutil
    fc = shutil.which("gfortran")
    return ("gfortran found at " + fc + " (the Fortran library is not built by this bench)"
            if fc else "gfortran absent on this host: the reference's OpenMP Fortran path "
                       "cannot be built; the C translation (sequential per call) is timed")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--plain-eps", type=float, default=1e-12,
                    help="eps of the all-FP64 plain comparison run")
    ap.add_argument("--accuracy-sample", type=int, default=10000)
    ap.add_argument("--ns", type=int, default=NS_DEFAULT)
    ap.add_argument("--nt", type=int, default=NT_DEFAULT)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--cpu-sample", type=int, default=100_000)
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--reference-full", action="store_true",
                    help="with --impl reference: also time one call of the full workload "
                         "(minutes on one core)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the library's default leaf capacity and M2L form")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (c1, c3, c4)")
    ap.add_argument("--configs", default="c1,c3,c4",
                    help="which of the other configurations to run (comma list)")
    ap.add_argument("--c4-points", type=int, default=2_000_000,
                    help="sources of the Helmholtz configuration (2e6 as named; smaller for "
                         "profiler captures)")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-baseline", type=int, default=2000,
                    help="requests of the one-at-a-time FP64 baseline (a prefix of the stream)")
    ap.add_argument("--serve-slots", type=int, default=6)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    import fmm2d_c_translation_b200 as fm

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if ws > 1:
            dist.barrier()

    L = fm.lib()
    L.fmm2d_b200_launch_count.restype = ctypes.c_ulonglong
    L.fmm2d_b200_set_precision({"auto": 0, "fp64": 1, "mixed": 2}[args.precision])
    stream = torch.cuda.current_stream()
    L.fmm2d_b200_set_stream(ctypes.c_void_p(stream.cuda_stream))

    ns, nt = args.ns, args.nt
    src, trg, q, d, v = make_inputs(ns, nt, 7 + rank)
    dev = torch.device("cuda", local)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    d_src, d_trg = t(src).to(dev), t(trg).to(dev)
    d_q = t(q.view(np.float64)).to(dev)
    d_d = t(d.view(np.float64)).to(dev)
    d_v = t(v).to(dev)
    d_pot = torch.zeros(2 * ns, dtype=torch.float64, device=dev)
    d_grad = torch.zeros(4 * ns, dtype=torch.float64, device=dev)
    d_pt = torch.zeros(2 * nt, dtype=torch.float64, device=dev)
    d_gt = torch.zeros(4 * nt, dtype=torch.float64, device=dev)
    eps = ctypes.c_double(args.eps)
    c_ns, c_nt = ctypes.c_int(ns), ctypes.c_int(nt)
    ier = ctypes.c_int(0)

    def ptr(x):
        return ctypes.c_void_p(x.data_ptr())

    def call(a):
        L.lfmm2d_st_cd_g_(ctypes.byref(eps), ctypes.byref(c_ns), ptr(a[0]),
                          ptr(a[2]), ptr(a[3]), ptr(a[4]), ptr(a[5]),
                          ptr(a[6]), ctypes.byref(c_nt), ptr(a[1]), ptr(a[7]),
                          ptr(a[8]), ctypes.byref(ier))
        if ier.value != 0:
            raise RuntimeError("lfmm2d_st_cd_g_ failed: " + fm.last_error())

    dev_args = (d_src, d_trg, d_q, d_d, d_v, d_pot, d_grad, d_pt, d_gt)

    # the library's autotuner picks the leaf capacity and M2L form of the
    # mixed path for this workload's order on its own points (untimed)
    tuned = None
    mixed_run = args.precision == "mixed" or (args.precision == "auto" and args.eps >= 0.5e-6)
    if mixed_run and not args.no_autotune:
        nd_, fm_, ms_ = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
        t0 = time.perf_counter()
        L.fmm2d_b200_autotune.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, P,
                                          ctypes.c_int, P, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, P, P, P]
        ier_t = L.fmm2d_b200_autotune(0, args.eps, ns, ptr(d_src), nt, ptr(d_trg), 1, 1, 2, 2,
                                      ctypes.byref(nd_), ctypes.byref(fm_), ctypes.byref(ms_))
        torch.cuda.synchronize()
        if ier_t == 0:
            tuned = {"leaf_capacity": nd_.value,
                     "m2l_form": ["window", "tile", "simt"][fm_.value],
                     "best_ms": ms_.value, "tuning_s": time.perf_counter() - t0,
                     "grid": "leaf capacity {12..64} x M2L form {window, tile, simt}"}

    def timed(a, steps, profile=False):
        L.fmm2d_b200_set_profiling(1 if profile else 0)
        evs = []
        prof = []
        buf = ctypes.create_string_buffer(4096)
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call(a)
            e1.record(stream)
            evs.append((e0, e1))
            if profile:
                L.fmm2d_b200_last_profile(buf, len(buf))
                prof.append(parse_profile(buf.value.decode()))
        torch.cuda.synchronize()
        L.fmm2d_b200_set_profiling(0)
        return [a_.elapsed_time(b_) for a_, b_ in evs], prof

    # ---- device-resident ----
    prec_code = {"auto": 0, "fp64": 1, "mixed": 2}

    def measure(precision, eps_value=None):
        eps.value = args.eps if eps_value is None else eps_value
        L.fmm2d_b200_set_precision(prec_code[precision])
        for _ in range(args.warmup):
            call(dev_args)
        torch.cuda.synchronize()
        barrier()
        clocks = ClockSampler(local)
        clocks.start()
        torch.cuda.synchronize()
        barrier()
        clocks.mark()
        n0 = L.fmm2d_b200_launch_count()
        ms, prof = timed(dev_args, args.steps, profile=True)
        n1 = L.fmm2d_b200_launch_count()
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        eps.value = args.eps
        t = max_over_ranks(sum(ms) / len(ms), ws, dev)
        return t, prof, clk, int(n1 - n0)

    def accuracy(precision, eps_value=None):
        """relative l2 errors at sampled targets vs the GPU FP64 direct sum"""
        eps.value = args.eps if eps_value is None else eps_value
        L.fmm2d_b200_set_precision(prec_code[precision])
        call(dev_args)
        eps.value = args.eps
        torch.cuda.synchronize()
        m = min(args.accuracy_sample, nt)
        idx = np.random.default_rng(99).choice(nt, m, replace=False)
        sub = torch.from_numpy(np.ascontiguousarray(trg[idx])).to(dev)
        pot = torch.zeros(2 * m, dtype=torch.float64, device=dev)
        grad = torch.zeros(4 * m, dtype=torch.float64, device=dev)
        ierd = L.fmm2d_b200_l2d_direct(1, ns, ptr(d_src), 1, ptr(d_q), 1, ptr(d_d),
                                       ptr(d_v), m, ptr(sub), 2, ptr(pot), ptr(grad),
                                       None, ctypes.c_double(1e-300))
        if ierd != 0:
            raise RuntimeError(fm.last_error())
        torch.cuda.synchronize()
        ix = torch.from_numpy(idx).to(dev)
        got_p = d_pt.view(-1, 2)[ix]
        got_g = d_gt.view(-1, 4)[ix]
        rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
        return {"pottarg_rel_l2": rel(got_p, pot.view(-1, 2)),
                "gradtarg_rel_l2": rel(got_g, grad.view(-1, 4)), "targets": m}

    t_step, prof, clk, nlaunch = measure(args.precision)
    value = whole_job_rate(ns + nt, ws, t_step)
    fp64 = None
    if args.precision != "fp64" and not args.no_fp64_compare:
        # the plain form of the workload: all-FP64 at eps = plain_eps
        t64, prof64, clk64, _ = measure("fp64", args.plain_eps)
        ph64 = {}
        for p_ in prof64:
            for k, v_ in p_.items():
                if not k.startswith("#"):
                    ph64.setdefault(k, []).append(v_)
        fp64 = {"value": ws * (ns + nt) / (t64 * 1e-3), "unit": "points/s",
                "eps": args.plain_eps, "precision": "fp64",
                "ms_per_step": t64, "speedup_of_headline": t64 / t_step,
                "phase_ms": {k: round(sum(v_) / len(v_), 4) for k, v_ in ph64.items()}}
    acc = None
    if rank == 0 and args.accuracy_sample > 0 and nt > 0:
        acc = {"sample": f"{min(args.accuracy_sample, nt)} random targets vs GPU FP64 direct sum over all sources",
               args.precision: accuracy(args.precision)}
        if fp64 is not None:
            acc[f"fp64_eps{args.plain_eps:g}"] = accuracy("fp64", args.plain_eps)
    L.fmm2d_b200_set_precision(prec_code[args.precision])

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        pin = lambda x: x.cpu().pin_memory()
        h_args = tuple(pin(x) for x in dev_args)
        for _ in range(max(1, args.warmup - 1)):
            call(h_args)
        torch.cuda.synchronize()
        barrier()
        ms_e2e, _ = timed(h_args, args.steps)
        barrier()
        te = max_over_ranks(sum(ms_e2e) / len(ms_e2e), ws, dev)
        h2d = sum(x.numel() * 8 for x in h_args[:5])
        d2h = sum(x.numel() * 8 for x in h_args[5:])
        e2e = {"value": ws * (ns + nt) / (te * 1e-3), "unit": "points/s",
               "ms_per_step": te, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h}

    if ws > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    # ---- roofline of the dominant phase ----
    phases = {}
    for p_ in prof:
        for k, v_ in p_.items():
            phases.setdefault(k, []).append(v_)
    avg = {k: sum(v_) / len(v_) for k, v_ in phases.items()}
    counts = {k[1:]: v_ for k, v_ in avg.items() if k.startswith("#")}
    times = {k: v_ for k, v_ in avg.items() if not k.startswith("#")}
    dom = max(times, key=times.get) if times else None
    peaks, peak_kind = read_peaks()
    ndc = counts.get("ndc", 2)
    pterm = counts.get("nterms", 18)
    mixed = args.precision == "mixed" or (args.precision == "auto" and args.eps >= 0.5e-6)
    pipe = "fp32" if mixed else "fp64"
    pk_pipe = measure_fp32_peak(L) if mixed else measure_fp64_peak(L)
    entries = {}
    if times.get("m2l"):
        # F_M2L = 8 * list-2 pairs * (p+1)^2 * nd_c
        f_m2l = 8.0 * counts.get("m2l_pairs", 0) * (pterm + 1) ** 2 * ndc
        ach = f_m2l / (times["m2l"] * 1e-3) / 1e12
        if mixed:
            # the tcgen05 kind::tf32 rate / 3: a TF32x3 product issues three MMAs
            tf32 = measure_tf32_peak(L)
            pk = tf32 / 3.0 if tf32 else None
            entries["m2l"] = {
                "kernel": "m2l phase (m2l_win_kernel tcgen05 TF32x3 on dense levels, "
                          "m2l_tc_kernel slot tables on sparse levels, FP32 leading rows)",
                "bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk if pk else None, "tf32_peak_tflops": tf32,
                "peak_source": "tcgen05 kind::tf32 microbenchmark on this GPU "
                               "(fmm2d_b200_tf32_peak_tflops), divided by 3",
                "flops_per_launch": f_m2l}
        else:
            entries["m2l"] = {
                "kernel": "m2l phase (m2l_dmma_kernel, FP64 DMMA)", "bound": "fp64",
                "achieved": ach, "peak": pk_pipe, "unit": "TFLOP/s",
                "frac": ach / pk_pipe if pk_pipe else None,
                "peak_source": "FP64 FMA microbenchmark on this GPU "
                               "(fmm2d_b200_fp64_peak_tflops)",
                "flops_per_launch": f_m2l}
    if times.get("p2p"):
        # F_P2P = pairs * (10 + nd_c * sum_out w), charge and dipole, pot + grad
        pairs = counts.get("p2p_pairs_src", 0) + counts.get("p2p_pairs_targ", 0)
        f_p2p = pairs * (10 + ndc * 20)
        ach = f_p2p / (times["p2p"] * 1e-3) / 1e12
        entries["p2p"] = {
            "kernel": "p2p phase (p2p_flat_kernel)" if mixed else "p2p phase (p2p_kernel)",
            "bound": pipe, "achieved": ach, "peak": pk_pipe, "unit": "TFLOP/s",
            "frac": ach / pk_pipe if pk_pipe else None,
            "peak_source": f"{pipe.upper()} FMA microbenchmark on this GPU "
                           f"(fmm2d_b200_{pipe}_peak_tflops); the kernel runs on the CUDA-core "
                           f"{pipe.upper()} pipe",
            "flops_per_launch": f_p2p}
    # DRAM bytes per launch of the dominant kernel from the ncu capture of the
    # same kernel at 2e6 + 2e6 points, scaled by the points (the traffic
    # grows with the boxes and points in proportion)
    tr = TRAFFIC_2E6.get(("mixed" if mixed else "fp64", dom))
    if tr is not None:
        entries[dom]["traffic"] = tr[0] * (ns + nt) / 4e6
        entries[dom]["traffic_source"] = tr[1]
    elif dom in entries:
        entries[dom]["traffic"] = None
    if dom in entries:
        roof = entries[dom]
    elif dom is not None:
        # memory-bound phases: compulsory bytes of the whole evaluation
        byts = (ns * (16 + 16 * ndc * 2 + 16) + nt * 16 +
                (ns + nt) * 16 * ndc * 3)
        ach = byts / (times[dom] * 1e-3) / 1e9
        pk = peaks.get("hbm_gbs")
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": pk,
                "unit": "GB/s", "frac": ach / pk if pk else None, "traffic": None}
    else:
        roof = None
    if roof is not None:
        roof["peak_file"] = peak_kind
        roof["hbm_peak_gbs"] = peaks.get("hbm_gbs")
        roof["phase_ms"] = {k: round(v_, 4) for k, v_ in times.items()}
        roof["counts"] = counts
    roof_other = {k: v_ for k, v_ in entries.items() if k != dom}

    configs = None
    if not args.no_configs and ws == 1:
        configs = measure_configs(fm, L, args)
        L.fmm2d_b200_set_precision(prec_code[args.precision])

    serving = None
    if args.serve_requests > 0:
        L.fmm2d_b200_reset_stream()
        try:
            serving = measure_serving(fm, args)
        except RuntimeError as e:
            serving = {"error": str(e)}

    cpu = None
    if not args.no_cpu_baseline and ws == 1:
        cpu = cpu_baseline_sample(args)

    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.precision != "fp64" else "f64", "data": "synthetic",
        "config": {"workload": f"lfmm2d_st_cd_g uniform {ns}+{nt} points eps {args.eps:g}",
                   "precision": args.precision, "ns": ns, "nt": nt,
                   "eps": args.eps, "parallelism": f"replicas{ws}",
                   "l2": "inputs 0.8 GB > L2; no flush"},
        "roofline": roof, "roofline_other_phases": roof_other, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": nlaunch, "clocks": clk, "fp64_plain": fp64,
        "accuracy": acc, "serving": serving, "configs": configs, "autotune": tuned,
    }
    print(json.dumps(line))
    return 0


def serving_stream(n_req, seed=2025):
    """The serving configuration's request mix: list of dicts."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n_req):
        n = int(round(10 ** rng.uniform(3.0, 6.0)))
        helm = rng.random() < 0.3
        reqs.append(dict(kernel="h" if helm else "l", n=n,
                         eps=1e-6 if helm else float(rng.choice([1e-3, 1e-6, 1e-9])),
                         zk=float(rng.uniform(1.0, 50.0)) if helm else 0.0,
                         blobs=bool(rng.random() < 0.5), off=int(rng.integers(0, 1 << 30))))
    return reqs


def measure_serving(fm, args):
    nmax = 1_000_000
    rng = np.random.default_rng(77)
    uni = np.asfortranarray(rng.random((2, nmax)))
    centers = rng.random((2, 32))
    blob = centers[:, rng.integers(0, 32, nmax)] + 0.01 * rng.standard_normal((2, nmax))
    blob = np.asfortranarray(np.clip(blob, 0.0, 1.0))
    chg = rng.standard_normal(nmax) + 1j * rng.standard_normal(nmax)
    reqs = serving_stream(args.serve_requests)

    def build(r, precision=0):
        n = r["n"]
        o = r["off"] % (nmax - n + 1)
        pts = (blob if r["blobs"] else uni)[:, o:o + n]
        return fm.make_request(r["kernel"], eps=r["eps"], sources=pts, charges=chg[o:o + n],
                               pg=2, zk=r["zk"], precision=precision)

    def run(stream, slots, precision, rate=None):
        """Submits `stream` (Poisson at `rate` req/s, or all at once);
        returns (wall s, latencies ms, points)."""
        srv = fm.Server(slots=slots, hbm_budget=args.serve_budget_gb * 1e9)
        lat = [None] * len(stream)
        tickets = [None] * len(stream)
        done = threading.Semaphore(0)
        failed = []

        def waiter():
            for i in range(len(stream)):
                done.acquire()
                ier, tms = srv.wait(tickets[i])
                if ier != 0:
                    failed.append((i, ier, fm.last_error()))
                lat[i] = tms[2]

        th = threading.Thread(target=waiter)
        th.start()
        arr = np.cumsum(np.random.default_rng(5).exponential(1.0 / rate, len(stream))) \
            if rate else np.zeros(len(stream))
        t0 = time.perf_counter()
        for i, r in enumerate(stream):
            dt = arr[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            req, keep = build(r, precision)
            tickets[i] = srv.submit(req, keep)
            done.release()
        th.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        if failed:
            i, ier, msg = failed[0]
            raise RuntimeError(f"{len(failed)} serving requests failed; request {i}: "
                               f"ier={ier} {msg}")
        return wall, lat, sum(r["n"] for r in stream), st

    # warm the pool and the code paths
    run(reqs[:20], args.serve_slots, 0)
    burst = reqs[: min(len(reqs), 300)]
    wall_b, _, pts_b, st_b = run(burst, args.serve_slots, 0)
    cap = len(burst) / wall_b
    rate = 0.7 * cap
    wall, lat, pts, st = run(reqs, args.serve_slots, 0, rate=rate)
    lat = np.array(lat)
    base = reqs[: min(len(reqs), args.serve_baseline)]
    # the baseline runs one request at a time: no batching either
    os.environ["FMM2D_B200_SERVE_BATCH"] = "0"
    try:
        wall1, lat1, pts1, _ = run(base, 1, 1)
    finally:
        os.environ.pop("FMM2D_B200_SERVE_BATCH", None)
    return {
        "requests": len(reqs), "slots": args.serve_slots,
        "hbm_budget_gb": args.serve_budget_gb,
        "arrival": f"Poisson at {rate:.1f} req/s (70% of the {cap:.1f} req/s burst capacity)",
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "mean_ms": float(lat.mean()), "throughput_req_s": len(reqs) / wall,
        "throughput_points_s": pts / wall, "burst_points_s": pts_b / wall_b,
        "peak_running": st["peak_running"], "peak_budget_gb": st["peak_bytes"] / 1e9,
        "batched_requests": st.get("batched", 0),
        "burst_batched_requests": st_b.get("batched", 0),
        "batching_note": "small lfmm2d requests of one kind are batched when they meet in the "
                         "queue: rarely at 70% load (short queues), often in the saturating burst; "
                         "Helmholtz requests carry their own zk (tables) and are not batched",
        "one_at_a_time_fp64": {"requests": len(base), "points_s": pts1 / wall1,
                               "sample": "the first requests of the same stream (one at a time "
                                         "they take about 8 ms each; all 20,000 would hold the GPU "
                                         "for minutes)",
                               "req_s": len(base) / wall1,
                               "p50_ms": float(np.percentile(lat1, 50))},
        "points": "N log-uniform [1e3, 1e6], uniform or Gaussian blobs, host arrays",
    }


def measure_configs(fm, L, args):
    """The other configurations the reference's FMM is quoted on, each timed
    device-resident through the C ABI (CUDA events, 3 warm-up + 3 timed
    calls) with its accuracy against the GPU FP64 direct sum on sampled
    points:
      c1 lfmm2d_s_c_g, 1e5 uniform sources, eps 1e-6 (with the reference's
         C translation on one host core for the same call);
      c3 lfmm2d_st_d_p on the starfish r = 1 + 0.3 cos 5t: 4e6 sources with
         outward normals as dipole vectors and real N(0,1) dipole strengths,
         4e6 targets at normal distance 10^U[-3,-1], eps 1e-9 (split-precision
         M2L, and all-FP64);
      c4 hfmm2d_s_cd_p, 2e6 uniform sources, zk = 200, eps 1e-6 (mixed: M2L as
         TF32x3 contractions on the tensor cores; also timed all-FP64)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ptr = lambda x: ctypes.c_void_p(x.data_ptr())
    ier = ctypes.c_int(0)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import pointsets as ps

    def timed(f, reps=3, warm=3):
        for _ in range(warm):
            f()
        torch.cuda.synchronize()
        L.fmm2d_b200_set_profiling(1)
        buf = ctypes.create_string_buffer(4096)
        ms = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            f()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        L.fmm2d_b200_last_profile(buf, len(buf))
        L.fmm2d_b200_set_profiling(0)
        prof = parse_profile(buf.value.decode())
        return min(ms), prof

    def check():
        if ier.value != 0:
            raise RuntimeError(fm.last_error())

    out = {}
    L.fmm2d_b200_set_precision(0)
    want = set(c for c in args.configs.split(",") if c)
    if "c1" in want:
        # ---- c1 ----
        rng = np.random.default_rng(101)
        ns = 100_000
        src = rng.random((ns, 2))
        q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
        d_src, d_q = T(src), T(q.view(np.float64))
        d_pot = torch.zeros(2 * ns, dtype=torch.float64, device=dev)
        d_grad = torch.zeros(4 * ns, dtype=torch.float64, device=dev)
        eps = ctypes.c_double(1e-6)
        cns = ctypes.c_int(ns)

        def c1():
            L.lfmm2d_s_c_g_(ctypes.byref(eps), ctypes.byref(cns), ptr(d_src), ptr(d_q), ptr(d_pot),
                            ptr(d_grad), ctypes.byref(ier))
            check()

        ms, prof = timed(c1)
        m = 1000
        sub = T(src[:m])
        pot = torch.zeros(2 * m, dtype=torch.float64, device=dev)
        grad = torch.zeros(4 * m, dtype=torch.float64, device=dev)
        # (thresh^2 must stay above zero to skip each sampled source's own pair)
        L.fmm2d_b200_l2d_direct(1, ns, ptr(d_src), 1, ptr(d_q), 0, None, None, m, ptr(sub), 2,
                                ptr(pot), ptr(grad), None, ctypes.c_double(1e-150))
        torch.cuda.synchronize()
        c1r = {"workload": "lfmm2d_s_c_g uniform 1e5 eps 1e-6 (auto: mixed)", "ms": ms,
               "phase_ms": {k: round(v, 3) for k, v in prof.items() if not k.startswith("#")},
               "points_s": ns / (ms * 1e-3),
               "pot_rel_l2": rel(d_pot.view(-1, 2)[:m], pot.view(-1, 2)),
               "grad_rel_l2": rel(d_grad.view(-1, 4)[:m], grad.view(-1, 4)),
               "accuracy_sample": f"{m} sources vs GPU FP64 direct sum"}
        import refimpl
        if refimpl.have_ref():
            R = refimpl.ref()
            hp, hg = np.zeros(ns, complex), np.zeros((ns, 2), complex)
            t0 = time.perf_counter()
            R.lfmm2d_s_c_g_(ctypes.byref(eps), ctypes.byref(cns), src.ctypes.data_as(P),
                            q.ctypes.data_as(P), hp.ctypes.data_as(P), hg.ctypes.data_as(P),
                            ctypes.byref(ier))
            tr = time.perf_counter() - t0
            c1r["reference_1core_ms"] = tr * 1e3
            c1r["vs_reference_1core"] = tr * 1e3 / ms
            c1r["pot_rel_l2_vs_reference"] = float(np.linalg.norm(
                d_pot.view(-1, 2).cpu().numpy().view(complex).ravel() - hp) / np.linalg.norm(hp))
            gg = d_grad.view(-1, 4).cpu().numpy().view(complex).reshape(ns, 2)
            c1r["grad_rel_l2_vs_reference"] = float(np.linalg.norm(gg - hg) / np.linalg.norm(hg))
            # the reference FMM's own errors at the same eps, same sampled sources
            dp = pot.view(-1, 2).cpu().numpy().view(complex).ravel()
            dg = grad.view(-1, 4).cpu().numpy().view(complex).reshape(m, 2)
            c1r["reference_pot_rel_l2"] = float(np.linalg.norm(hp[:m] - dp) / np.linalg.norm(dp))
            c1r["reference_grad_rel_l2"] = float(np.linalg.norm(hg[:m] - dg) / np.linalg.norm(dg))
        out["c1"] = c1r
    if "c3" in want:
        # ---- c3 ----
        n3 = 4_000_000
        x, nrm = ps.starfish(n3, 0)
        y = ps.near_curve_targets(n3, 1)
        ds = np.random.default_rng(3).standard_normal(n3) + 0j
        d_src, d_trg = T(x.T), T(y.T)
        d_ds, d_nv = T(ds.view(np.float64)), T(nrm.T)
        d_pot = torch.zeros(2 * n3, dtype=torch.float64, device=dev)
        d_pt = torch.zeros(2 * n3, dtype=torch.float64, device=dev)
        eps3 = ctypes.c_double(1e-9)
        c3n = ctypes.c_int(n3)

        def c3():
            L.lfmm2d_st_d_p_(ctypes.byref(eps3), ctypes.byref(c3n), ptr(d_src), ptr(d_ds),
                             ptr(d_nv), ptr(d_pot), ctypes.byref(c3n), ptr(d_trg), ptr(d_pt),
                             ctypes.byref(ier))
            check()

        m = 10000
        idx = np.random.default_rng(5).choice(n3, m, replace=False)
        sub = T(y.T[idx])
        pot = torch.zeros(2 * m, dtype=torch.float64, device=dev)
        L.fmm2d_b200_l2d_direct(1, n3, ptr(d_src), 0, None, 1, ptr(d_ds), ptr(d_nv), m, ptr(sub), 1,
                                ptr(pot), None, None, ctypes.c_double(1e-300))
        torch.cuda.synchronize()
        # split-precision M2L (FP64 triangle + TF32x3 tail on the tensor
        # cores), then the same call all-FP64
        L.fmm2d_b200_set_precision(3)
        ms, prof = timed(c3)
        err_split = rel(d_pt.view(-1, 2)[T(idx)], pot.view(-1, 2))
        L.fmm2d_b200_set_precision(1)
        ms64, prof64 = timed(c3)
        err64 = rel(d_pt.view(-1, 2)[T(idx)], pot.view(-1, 2))
        L.fmm2d_b200_set_precision(0)
        out["c3"] = {"workload": "lfmm2d_st_d_p starfish 4e6 + 4e6 near-curve targets eps 1e-9 "
                                 "(split: FP64 passes, M2L terms of total order >= "
                                 f"{int(prof.get('#m2l_split_nt', 0))} as TF32x3 on the tensor cores)",
                     "ms": ms, "points_s": 2 * n3 / (ms * 1e-3),
                     "nlevels": prof.get("#nlevels"), "nboxes": prof.get("#nboxes"),
                     "phase_ms": {k: round(v, 3) for k, v in prof.items() if not k.startswith("#")},
                     "pottarg_rel_l2": err_split,
                     "accuracy_sample": f"{m} targets vs GPU FP64 direct sum",
                     "fp64": {"ms": ms64, "points_s": 2 * n3 / (ms64 * 1e-3),
                              "pottarg_rel_l2": err64,
                              "phase_ms": {k: round(v, 3) for k, v in prof64.items()
                                           if not k.startswith("#")}}}
        del d_src, d_trg, d_ds, d_nv, d_pot, d_pt
    if "c4" in want:
        # ---- c4 ----
        n4 = args.c4_points
        rng = np.random.default_rng(404)
        src = rng.random((n4, 2))
        q = rng.standard_normal(n4) + 1j * rng.standard_normal(n4)
        dd = rng.standard_normal(n4) + 1j * rng.standard_normal(n4)
        th = rng.uniform(0, 2 * np.pi, n4)
        v = np.stack([np.cos(th), np.sin(th)], axis=1)
        d_src, d_q, d_d, d_v = T(src), T(q.view(np.float64)), T(dd.view(np.float64)), T(v)
        d_pot = torch.zeros(2 * n4, dtype=torch.float64, device=dev)
        zk = np.array([200.0, 0.0])
        eps4 = ctypes.c_double(1e-6)
        c4n = ctypes.c_int(n4)

        def c4():
            L.hfmm2d_s_cd_p_(ctypes.byref(eps4), zk.ctypes.data_as(P), ctypes.byref(c4n), ptr(d_src),
                             ptr(d_q), ptr(d_d), ptr(d_v), ptr(d_pot), ctypes.byref(ier))
            check()

        L.fmm2d_b200_set_precision(1)
        ms64, prof64 = timed(c4)
        L.fmm2d_b200_set_precision(0)
        ms, prof = timed(c4)
        m = 1000
        sub = T(src[:m])
        pot = torch.zeros(2 * m, dtype=torch.float64, device=dev)
        L.fmm2d_b200_h2d_direct(1, zk.ctypes.data_as(P), n4, ptr(d_src), 1, ptr(d_q), 1, ptr(d_d),
                                ptr(d_v), m, ptr(sub), 1, ptr(pot), None, None,
                                ctypes.c_double(1e-150))
        torch.cuda.synchronize()
        h_ms = prof.get("h_m2l", 0.0)
        tf32 = measure_tf32_peak(L)
        m2l_ach = prof.get("#h_m2l_flops", 0.0) / (h_ms * 1e-3) / 1e12 if h_ms else None
        out["c4"] = {"workload": f"hfmm2d_s_cd_p uniform {n4:.0e} zk 200 eps 1e-6 "
                                 "(auto: mixed, TF32x3 tensor-core M2L on levels of order <= 23)",
                     "ms": ms, "points_s": n4 / (ms * 1e-3),
                     "phase_ms": {k: round(v, 3) for k, v in prof.items() if not k.startswith("#")},
                     "counts": {k[1:]: v for k, v in prof.items() if k.startswith("#")},
                     "pot_rel_l2": rel(d_pot.view(-1, 2)[:m], pot.view(-1, 2)),
                     "accuracy_sample": f"{m} sources vs GPU FP64 direct sum",
                     "m2l_roofline": {
                         "bound": "tensor", "unit": "TFLOP/s",
                         "achieved": m2l_ach,
                         "peak": tf32 / 3.0 if tf32 else None,
                         "frac": (m2l_ach / (tf32 / 3.0)) if (m2l_ach and tf32) else None,
                         "peak_source": "tcgen05 kind::tf32 microbenchmark "
                                        "(fmm2d_b200_tf32_peak_tflops) / 3: a TF32x3 product "
                                        "issues three MMAs",
                         "tf32_peak_tflops": tf32,
                         "flops": "F_M2L = 8 sum_l list2_pairs_l (2 p_l + 1)^2 nd over the whole "
                                  "M2L phase (tensor-core and FP64 levels)"},
                     "fp64": {"ms": ms64, "points_s": n4 / (ms64 * 1e-3),
                              "phase_ms": {k: round(v, 3) for k, v in prof64.items()
                                           if not k.startswith("#")}}}
    return out


def measure_fp32_peak(L):
    L.fmm2d_b200_fp32_peak_tflops.restype = ctypes.c_double
    return L.fmm2d_b200_fp32_peak_tflops()


def measure_tf32_peak(L):
    L.fmm2d_b200_tf32_peak_tflops.restype = ctypes.c_double
    return L.fmm2d_b200_tf32_peak_tflops()


def measure_fp64_peak(L):
    L.fmm2d_b200_fp64_peak_tflops.restype = ctypes.c_double
    return L.fmm2d_b200_fp64_peak_tflops()


if __name__ == "__main__":
    sys.exit(main())
