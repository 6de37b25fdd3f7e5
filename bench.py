#!/usr/bin/env python3
"""Benchmark of the B200 F-J transform on the large-array noise workload.

Workload (one "step"): ccfj fj_noise, itype=1 (linear-interpolation
integral), func=0 (Bessel basis) on 19,900 station pairs (all pairs of 200
stations at seeded uniform positions in a 300 x 300 km box), nf = 2048
frequencies over 0.005-2 Hz, nc = 1000 phase velocities over 500-5000 m/s;
complex64 spectra from the c(f) law with a first overtone and sigma = 0.2
noise (tests/cases.py). Metric: F-J terms per second, terms = nf * nc * npairs.

  value   inputs resident in HBM; one step = the full device transform
          (gather by the sort permutation, interval preparation, the FP32
          station-amortised kernel, per-frequency normalisation)
  e2e     the same metric through the public API ccfj.fj_noise on host
          numpy arrays (host->device copy of the spectra and device->host copy
          of the result inside the timed region)

  --impl reference   times the reference's own CPU implementation
          (src/ccfj.pyx over src/FJcpu.cpp with OpenMP, built into
          oracle/_ref by `make -C oracle`) on a frequency subset of the same
          workload, on all host cores.

Multi-GPU (torchrun): every rank transforms its own copy of the workload (the
transform shards by frequency or by data set with no exchange: weak scaling);
time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
import warnings

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "cc-fjpy_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))

METRIC = "F-J terms/s (nf·nc·npairs), FP32/batched vs FP64 GPU form at ≤1e-4 rel err"
NPAIRS, NF, NC = 19900, 2048, 1000
FLOPS_PER_TERM_ITYPE1 = 128  # algorithmic FLOPs per (f, c, pair) term, FMA = 2


def workload(seed=2):
    import cases
    rng = np.random.default_rng(seed)
    xy = rng.uniform(0.0, 3e5, (200, 2))
    i, j = np.triu_indices(200, k=1)
    r = np.hypot(xy[i, 0] - xy[j, 0], xy[i, 1] - xy[j, 1])
    f = np.linspace(0.005, 2.0, NF)
    c = np.linspace(500.0, 5000.0, NC)
    uf = cases.noise_spectra(rng, r, f, sigma=0.2, overtone=True)
    return uf, r, f, c


def config_dict():
    return {"workload": "fj_noise large array: %d pairs (200 stations, 300x300 km), nf=%d over "
                        "0.005-2 Hz, nc=%d over 500-5000 m/s, itype=1, func=0" % (NPAIRS, NF, NC),
            "npairs": NPAIRS, "nf": NF, "nc": NC, "itype": 1, "func": 0,
            "l2": "inputs larger than L2 (326 MB complex64 spectra + 326 MB interval data)",
            "parallelism": "one GPU per rank, independent workloads"}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [ln.split(",") for ln in self.f.read().strip().splitlines() if ln.count(",") >= 5]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(x[0]) for x in rows if x[0].strip().replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for x in rows for k in range(4) if "Active" in x[2 + k]
                          and "Not" not in x[2 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].strip().replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_smi_index(dev):
    import torch
    p = torch.cuda.get_device_properties(dev)
    try:
        return "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
    except AttributeError:
        return dev


# ------------------------------------------------------------ CPU baseline
def reference_module():
    ref_dir = os.path.join(REPO, "oracle", "_ref")
    if ref_dir not in sys.path:
        sys.path.insert(0, ref_dir)
    import ccfj_ref  # the reference's Cython module over FJcpu.cpp
    return ccfj_ref


def cpu_reference_step(ref, uf, r, f, c, cols, threads):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        t0 = time.perf_counter()
        ref.fj_noise(uf[:, cols], r, c, f[cols], itype=1, func=0, num=threads)
        return time.perf_counter() - t0


def cpu_sample_columns(ref, uf, r, f, c, threads, target_s):
    """Evenly spaced frequency subset sized so that one call takes about
    target_s seconds (calibrated with a 2-column call)."""
    cols = np.linspace(0, NF - 1, 2).astype(int)
    t = cpu_reference_step(ref, uf, r, f, c, cols, threads)
    n = int(max(2, min(NF, round(2 * target_s / max(t, 1e-6)))))
    return np.unique(np.linspace(0, NF - 1, n).astype(int))


def cpu_baseline(uf, r, f, c):
    threads = os.cpu_count() or 1
    ref = reference_module()
    cols = cpu_sample_columns(ref, uf, r, f, c, threads, target_s=5.0)
    ts = [cpu_reference_step(ref, uf, r, f, c, cols, threads) for _ in range(3)]
    t = sum(ts)
    terms = 3 * len(cols) * NC * NPAIRS
    return {"value": terms / t, "unit": "terms/s", "cores": threads, "kind": "reference",
            "sample": "reference fj_noise (src/ccfj.pyx + src/FJcpu.cpp, OpenMP, %d threads) on %d "
                      "evenly spaced of the %d frequencies, all %d pairs and %d velocities, 3 calls "
                      "(%.1f s)" % (threads, len(cols), NF, NPAIRS, NC, t)}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    uf, r, f, c = workload()
    threads = os.cpu_count() or 1
    try:
        ref = reference_module()
    except ImportError as e:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built: %s" % e}))
        return 0
    cols = cpu_sample_columns(ref, uf, r, f, c, threads, target_s=3.0)
    for _ in range(args.warmup):
        cpu_reference_step(ref, uf, r, f, c, cols, threads)
    ts = [cpu_reference_step(ref, uf, r, f, c, cols, threads) for _ in range(args.steps)]
    t = sum(ts)
    value = args.steps * len(cols) * NC * NPAIRS / t
    sample = ("reference fj_noise on %d evenly spaced of %d frequencies (all %d pairs, %d "
              "velocities) per step" % (len(cols), NF, NPAIRS, NC))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "terms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)", "config": config_dict(),
        "cpu_baseline": {"value": value, "unit": "terms/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "terms/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))
    return 0


# -------------------------------------------------------------- our arm
def traffic_per_launch():
    """DRAM bytes of one launch of the main kernel from the committed ncu
    summary (profiles/fj_amortized_config2.md, line 'traffic_bytes_per_launch:')."""
    p = os.path.join(REPO, "profiles", "fj_amortized_config2.md")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def run_ours(args, rank, world):
    import torch
    import ccfj
    from ccfj import _lib

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lib = _lib.load()
    uf, r, f, c = workload()
    idx = np.argsort(r)
    rs = np.ascontiguousarray(r[idx], dtype=np.float32)
    s = torch.cuda.current_stream()
    sp = ctypes.c_void_p(s.cuda_stream)

    # device-resident inputs: complex64 spectra as float pairs (real part at
    # even offsets), the sort permutation, sorted distances, f, c
    d_u = torch.from_numpy(uf.view(np.float32)).cuda()
    d_perm = torch.from_numpy(idx.astype(np.int64)).cuda()
    d_r = torch.from_numpy(rs).cuda()
    d_f = torch.from_numpy(f.astype(np.float32)).cuda()
    d_c = torch.from_numpy(c.astype(np.float32)).cuda()
    d_out = torch.empty((NC, NF), dtype=torch.float32, device="cuda")

    def args_for(prec, nf=NF, out=d_out):
        a = _lib.FjArgs()
        a.struct_size = ctypes.sizeof(a)
        a.nr, a.nf, a.nc = NPAIRS, nf, NC
        a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, _lib.MODE_J, prec, 1, 1
        a.u[0] = d_u.data_ptr()
        a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * NF, NPAIRS, 2, nf, 1
        a.perm = d_perm.data_ptr()
        a.r, a.f, a.c, a.out = d_r.data_ptr(), d_f.data_ptr(), d_c.data_ptr(), out.data_ptr()
        return a

    a32 = args_for(_lib.PREC_FP32)

    def step():
        _lib.check(lib.ccfj_fj_v1(ctypes.byref(a32), sp))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_smi_index(dev))
    lib.ccfj_profile_enable(1)
    l0 = lib.ccfj_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    launches = lib.ccfj_launch_count() - l0
    clocks = sampler.stop()
    t = e0.elapsed_time(e1) / 1e3
    cnt = ctypes.c_int(0)
    kern_ms = lib.ccfj_profile_total_ms(ctypes.byref(cnt)) / max(cnt.value, 1)
    lib.ccfj_profile_enable(0)
    if dist:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    terms = NF * NC * NPAIRS
    value = world * terms * args.steps / t

    # end to end through the public API on host arrays
    for _ in range(max(1, args.warmup // 2)):
        ccfj_out = _quiet(ccfj.fj_noise, uf, r, c, f, itype=1, func=0)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2e_steps = max(2, min(args.steps, 5))
    w0 = time.perf_counter()
    e0.record()
    for _ in range(e2e_steps):
        ccfj_out = _quiet(ccfj.fj_noise, uf, r, c, f, itype=1, func=0)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    t_e2e = e0.elapsed_time(e1) / 1e3
    if dist:
        tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e = {"value": world * terms * e2e_steps / t_e2e, "unit": "terms/s",
           "h2d_bytes_per_step": int(uf.nbytes + rs.nbytes + idx.astype(np.int64).nbytes
                                     + 4 * (NF + NC)),
           "d2h_bytes_per_step": int(ccfj_out.nbytes), "wall_s_per_step": wall / e2e_steps}

    result = None
    if rank == 0:
        # accuracy and the FP64 comparators (outside the timed region)
        y32 = d_out.cpu().numpy()
        d64 = torch.empty_like(d_out)
        a64 = args_for(_lib.PREC_FP64, out=d64)
        t0 = time.perf_counter()
        _lib.check(lib.ccfj_fj_v1(ctypes.byref(a64), sp))
        torch.cuda.synchronize()
        y64 = d64.cpu().numpy()
        err = float(np.nanmax(np.abs(y32.astype(np.float64) - y64)))
        # plain FP64 form (the reference's loop structure) on a frequency subset
        nsub = 64
        d_pl = torch.empty((NC, nsub), dtype=torch.float32, device="cuda")
        apl = args_for(_lib.PREC_FP64_PLAIN, nf=nsub, out=d_pl)
        apl.u_ld = 2 * NF
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        _lib.check(lib.ccfj_fj_v1(ctypes.byref(apl), sp))
        ev1.record()
        torch.cuda.synchronize()
        plain_tps = nsub * NC * NPAIRS / (ev0.elapsed_time(ev1) / 1e3)
        peak = ctypes.c_double(0)
        _lib.check(lib.ccfj_fp32_peak_probe(sp, ctypes.byref(peak)))
        achieved = FLOPS_PER_TERM_ITYPE1 * terms / (kern_ms / 1e3) / 1e12
        traffic = traffic_per_launch()
        cpu = cpu_baseline(uf, r, f, c)
        result = {
            "metric": METRIC, "value": value, "unit": "terms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; spectra from the c(f) dispersion law)",
            "config": config_dict(), "e2e": e2e,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value,
                         "unit": "TFLOP/s", "frac": achieved / peak.value, "traffic": traffic,
                         "kernel": "fj_amortized_kernel<MODE_J, itype 1, float>",
                         "kernel_ms": kern_ms,
                         "flops_per_term": FLOPS_PER_TERM_ITYPE1,
                         "peak_source": "measured at bench time: FP32 FMA probe "
                                        "(ccfj_fp32_peak_probe); MEASURED_PEAKS.json has no FP32 "
                                        "figure"},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "accuracy": {"max_abs_err_vs_fp64_normalised": err,
                         "fp64_plain_terms_per_s": plain_tps,
                         "speedup_vs_fp64_plain": value / world / plain_tps},
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))
    return 0


def run_profile_case(args):
    """The device transform on the first 512 frequencies of the workload
    (19,900 pairs, 1000 velocities; 163 MB of spectra, 163 MB of station
    coefficients: larger than L2). With --profile-case hilbert, the func-1
    form: J of the spectra minus Y of their Hilbert transform along the
    512 columns."""
    import torch
    from ccfj import _lib
    lib = _lib.load()
    uf, r, f, c = workload()
    nf = 512
    idx = np.argsort(r)
    d_u = torch.from_numpy(uf.view(np.float32)).cuda()
    d_perm = torch.from_numpy(idx.astype(np.int64)).cuda()
    d_r = torch.from_numpy(np.ascontiguousarray(r[idx], dtype=np.float32)).cuda()
    d_f = torch.from_numpy(f.astype(np.float32)).cuda()
    d_c = torch.from_numpy(c.astype(np.float32)).cuda()
    d_out = torch.empty((NC, nf), dtype=torch.float32, device="cuda")
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nr, a.nf, a.nc = NPAIRS, nf, NC
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, _lib.MODE_J, 0, 1, 1
    if args.profile_case == "hilbert":
        a.mode, a.hilbert = _lib.MODE_J_MINUS_Y, 1
    a.u[0] = d_u.data_ptr()
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * NF, NPAIRS, 2, nf, 1
    a.perm = d_perm.data_ptr()
    a.r, a.f, a.c, a.out = d_r.data_ptr(), d_f.data_ptr(), d_c.data_ptr(), d_out.data_ptr()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(args.warmup + args.steps):
        _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))
    torch.cuda.synchronize()
    print("profile case done: %d transforms of %d x %d x %d" % (args.warmup + args.steps, NPAIRS,
                                                                 nf, NC))
    return 0


def run_cc_case(args):
    """Cross-correlation (ccfj.CC) on the reference example's day: 200
    stations x 345,600 samples at 4 Hz (276 MB of records), one-hour windows
    (14,400 samples) at 0.9 overlap (steplen 1439: 231 windows per station),
    1000 bins at fstride 3, all 19,900 pairs. Device-resident calls timed
    with CUDA events on the launching stream, and host-memory calls
    (ccfj.CC, copies included) timed on the wall clock. The records (276 MB)
    and the spectra the call writes and reads (378 MB) are larger than L2."""
    import time
    import torch
    import ccfj
    from ccfj import _cc, _lib
    lib = _lib.load()
    nsta, fs = 200, 4
    npts, fftlen, nf, fstride, overlap = 86400 * fs, 3600 * fs, 1000, 3, 0.9
    data = np.random.default_rng(7).standard_normal(nsta * npts, dtype=np.float32)
    se = np.tile([0, npts], nsta).astype(np.int32)
    pairs = ccfj.GetStationPairs(nsta)
    npairs = len(pairs) // 2
    a, keep, _ = _cc._prepare(npts, nsta, nf, fftlen, pairs, se, data, overlaprate=overlap,
                              fstride=fstride)
    d_data = torch.from_numpy(data).cuda()
    d_out = torch.empty((npairs, 2 * nf), dtype=torch.float32, device="cuda")
    a.device_ptrs, a.data, a.out_re = 1, d_data.data_ptr(), d_out.data_ptr()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    launches0 = lib.ccfj_launch_count()
    dev_s = _time_device(lambda: _lib.check(lib.ccfj_cc_v1(ctypes.byref(a), sp)), args.steps,
                         args.warmup)
    launches = (lib.ccfj_launch_count() - launches0) // (args.steps + args.warmup)
    for _ in range(args.warmup):
        ccfj.CC(npts, nsta, nf, fftlen, pairs, se, data, overlaprate=overlap, fstride=fstride)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ccfj.CC(npts, nsta, nf, fftlen, pairs, se, data, overlaprate=overlap, fstride=fstride)
    e2e_s = (time.perf_counter() - t0) / args.steps
    nshifts = 1 + (npts - fftlen) // int(a.steplen)   # every record covers the day
    windows = nshifts * nsta
    fft_flops = windows * 5.0 * fftlen * np.log2(fftlen)
    pair_flops = 8.0 * npairs * nf * nshifts
    peak = ctypes.c_double(0)
    _lib.check(lib.ccfj_fp32_peak_probe(sp, ctypes.byref(peak)))
    tflops = (fft_flops + pair_flops) / dev_s / 1e12
    print(json.dumps({
        "case": "cc", "unit": "ms per call", "device_ms": dev_s * 1e3, "e2e_ms": e2e_s * 1e3,
        "gpu_launches_per_call": int(launches),
        "algorithmic_tflops": tflops, "fp32_peak_tflops": peak.value,
        "frac_fp32": tflops / peak.value,
        "flops": {"fft": fft_flops, "pair_products": pair_flops},
        "config": {"workload": "CC, reference example day", "nsta": nsta, "npts": npts,
                   "fftlen": fftlen, "steplen": int(a.steplen), "windows": windows, "nf": nf,
                   "fstride": fstride, "npairs": npairs, "l2": "inputs larger than L2"},
        "data": "synthetic (seeded standard normal records)"}))
    return 0


# ------------------------------------------------- the other configurations
def _dev_args(lib_, torch, nr, nf, nc, itype, mode, u_ptr, u_ld, u_es, perm_ptr, r_t, f_t, c_t,
              out_t, u2_ptr=None, hilbert=0, ncols=None):
    from ccfj import _lib
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nr, a.nf, a.nc = nr, nf, nc
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = itype, mode, 0, 1, 1
    a.hilbert = hilbert
    a.u[0] = u_ptr
    a.u[1] = u2_ptr
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = u_ld, nr, u_es, ncols or nf, 1
    a.perm = perm_ptr or None
    a.r, a.f, a.c, a.out = r_t.data_ptr(), f_t.data_ptr(), c_t.data_ptr(), out_t.data_ptr()
    return a


def _time_device(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def _max_err(y32, y64, sample):
    e = np.abs(y32.astype(np.float64) - y64.astype(np.float64))
    return {"max_abs_err_vs_fp64_normalised": float(np.nanmax(e)),
            "nan_positions_equal": bool(np.array_equal(np.isnan(y32), np.isnan(y64))),
            "sample": sample}


def run_config(args):
    """Device-resident timing of the other workloads (one JSON line each; the
    headline bench line is the large-array noise workload, 2):
      1  small noise array: 200 pairs x 512 f x 300 c
      3  fj_earthquake: 500 traces x 8192 samples, rFFT on the GPU, nf 1024, 800 c
      4  MWFJ: 1000 traces x 16384 samples, 64 windows, nf 1024, 2000 c
      5  ragged batch: 512 subarrays (50-20000 pairs each), nf 1024, 500 c"""
    import torch
    import cases
    from ccfj import _lib, _batch, _eq
    lib = _lib.load()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cfg = args.config
    res = {"config_id": cfg, "unit": "terms/s", "dtype": "f32", "data": "synthetic (seeded)"}
    if cfg == 1:
        rng = np.random.default_rng(1)
        r = np.sort(rng.uniform(1e3, 5e4, 200))
        f = np.linspace(0.01, 1.0, 512)
        c = np.linspace(1000, 5000, 300)
        uf = cases.noise_spectra(rng, r, f, sigma=0.1)
        d = {k: torch.from_numpy(v).cuda() for k, v in dict(
            u=uf.view(np.float32), r=r.astype(np.float32), f=f.astype(np.float32),
            c=c.astype(np.float32)).items()}
        out = torch.empty((300, 512), device="cuda")
        a = _dev_args(lib, torch, 200, 512, 300, 1, 0, d["u"].data_ptr(), 1024, 2, None, d["r"],
                      d["f"], d["c"], out)
        t = _time_device(lambda: _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp)), args.steps,
                         args.warmup)
        y32 = out.cpu().numpy()
        a.precision = _lib.PREC_FP64
        _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))
        res.update(workload="fj_noise itype=1 func=0, 200 pairs x 512 f x 300 c", seconds=t,
                   value=200 * 512 * 300 / t,
                   accuracy=_max_err(y32, out.cpu().numpy(), "all 300 x 512"))
    elif cfg in (3, 4):
        if cfg == 3:
            rng = np.random.default_rng(3)
            ntr, npts, Fs, nf, nwin = 500, 8192, 20.0, 1024, 0
            r = np.exp(rng.uniform(np.log(1e4), np.log(2e6), ntr))
            c = np.linspace(2000, 5000, 800)
        else:
            rng = np.random.default_rng(4)
            ntr, npts, Fs, nf, nwin = 1000, 16384, 10.0, 1024, 64
            if getattr(args, "mwfj_small", False):
                nf, nwin = 256, 8
            r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e6), ntr))
            c = np.linspace(1500, 5000, 2000)
        u = cases.ricker_records(rng, r, npts, Fs)
        f = Fs * np.arange(nf) / npts
        nc = len(c)
        idx = np.argsort(r)
        d = {k: torch.from_numpy(v).cuda() for k, v in dict(
            u=u, perm=idx.astype(np.int64), r=r[idx].astype(np.float32), f=f.astype(np.float32),
            c=c.astype(np.float32)).items()}
        nw = max(nwin, 1)
        out = torch.empty((nw, nc, nf), device="cuda")
        a = _eq.EqArgs()
        a.struct_size = ctypes.sizeof(a)
        a.ntr, a.npts, a.nf, a.nc = ntr, npts, nf, nc
        a.itype, a.func, a.precision, a.normalize, a.device_ptrs, a.fstride = 1, 0, 0, 1, 1, 1
        a.func = getattr(args, "mwfj_func", 0)  # func 1 takes the CUDA-core MWFJ kernel
        a.nwin = nwin
        a.u, a.u_ld, a.u_rows = d["u"].data_ptr(), npts, ntr
        a.perm, a.r, a.f, a.c = d["perm"].data_ptr(), d["r"].data_ptr(), d["f"].data_ptr(), \
            d["c"].data_ptr()
        if nwin:
            L = rng.integers(200, 2001, size=(nwin, ntr))
            start = rng.integers(0, npts - L)
            n1, n2, dl = _eq._win_params(npts, Fs, start / Fs, (start + L) / Fs, 0.9)
            W = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.int32)).cuda()
                 for k, v in dict(n1=n1, n2=n2, dl=dl).items()}
            a.win_n1, a.win_n2, a.win_delta = W["n1"].data_ptr(), W["n2"].data_ptr(), \
                W["dl"].data_ptr()
        a.out = out.data_ptr()
        fn = lambda: _lib.check(lib.ccfj_fj_earthquake_v1(ctypes.byref(a), sp))  # noqa: E731
        t = _time_device(fn, max(1, args.steps // (4 if cfg == 4 else 1)), 1)
        terms = nw * nf * nc * ntr
        # FP64 station-amortised form on the same spectra (MWFJ: its first 4
        # windows, one transform per window)
        y32 = out.cpu().numpy()
        n64 = min(nw, 4)
        a.precision = _lib.PREC_FP64
        if nwin:
            a.nwin = n64
        _lib.check(lib.ccfj_fj_earthquake_v1(ctypes.byref(a), sp))
        y64 = out[:n64].cpu().numpy()
        res["accuracy"] = _max_err(y32[:n64], y64, "windows 0-%d" % (n64 - 1) if nwin else
                                   "all 800 x 1024")
        res.update(workload=("fj_earthquake itype=1 func=0 with device rFFT, 500 traces x 8192 "
                             "samples, nf=1024 bins, nc=800" if cfg == 3 else
                             "MWFJ itype=1 func=%d, 1000 traces x 16384 samples, %d windows, "
                             "nf=%d, nc=2000" % (a.func, nwin, nf)), seconds=t, value=terms / t)
    elif cfg == 5:
        rng = np.random.default_rng(5)
        nsets, nf, nc = (64 if getattr(args, "batch_small", False) else 512), 1024, 500
        counts = np.exp(rng.uniform(np.log(50), np.log(20000), nsets)).astype(np.int64)
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        total = int(off[-1])
        f = np.linspace(0.01, 1.0, nf)
        c = np.linspace(1000, 5000, nc)
        # spectra generated on the device (14 GB as complex64): c(f) law with
        # an overtone and sigma = 0.2 noise, as the large-array workload
        g = torch.Generator(device="cuda").manual_seed(5)
        r_t = (torch.rand(total, generator=g, device="cuda", dtype=torch.float64) * 299.5e3 + 500.0)
        f_t = torch.from_numpy(f).cuda()
        cf = 2000.0 + 1500.0 * torch.exp(-f_t / 0.2)
        U = torch.empty((total, 2 * nf), dtype=torch.float32, device="cuda")
        for s0 in range(0, total, 65536):
            rr = r_t[s0:s0 + 65536, None]
            ph = 2 * np.pi * f_t[None, :] * rr
            re = torch.special.bessel_j0(ph / cf) + 0.5 * torch.special.bessel_j0(ph / (cf + 800))
            n = rr.shape[0]
            U[s0:s0 + n, 0::2] = (re + 0.2 * torch.randn(n, nf, generator=g, device="cuda",
                                                        dtype=torch.float64)).float()
            U[s0:s0 + n, 1::2] = (0.2 * torch.randn(n, nf, generator=g, device="cuda",
                                                   dtype=torch.float64)).float()
        r_sorted = torch.empty(total, dtype=torch.float32, device="cuda")
        perm = torch.empty(total, dtype=torch.int64, device="cuda")
        for b in range(nsets):
            seg = r_t[off[b]:off[b + 1]]
            srt, ix = torch.sort(seg, stable=True)
            r_sorted[off[b]:off[b + 1]] = srt.float()
            perm[off[b]:off[b + 1]] = ix + int(off[b])
        d_off = torch.from_numpy(off).cuda()
        f32 = torch.from_numpy(f.astype(np.float32)).cuda()
        c32 = torch.from_numpy(c.astype(np.float32)).cuda()
        out = torch.empty((nsets, nc, nf), device="cuda")
        ba = _batch.BatchArgs()
        ba.struct_size = ctypes.sizeof(ba)
        ba.nsets, ba.nf, ba.nc = nsets, nf, nc
        ba.itype, ba.mode, ba.precision, ba.normalize, ba.device_ptrs = 1, 0, 0, 1, 1
        ba.use_graph = 1
        ba.offsets, ba.total_pairs = d_off.data_ptr(), total
        ba.r, ba.u[0] = r_sorted.data_ptr(), U.data_ptr()
        ba.u_ld, ba.u_rows, ba.u_es, ba.u_ncols, ba.fstride = 2 * nf, total, 2, nf, 1
        ba.perm, ba.f, ba.c, ba.out = perm.data_ptr(), f32.data_ptr(), c32.data_ptr(), \
            out.data_ptr()
        s_cap = torch.cuda.Stream()
        spc = ctypes.c_void_p(s_cap.cuda_stream)

        def batch_step():
            _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(ba), spc))

        with torch.cuda.stream(s_cap):
            t_batch = _time_device(batch_step, 2, 1)
        lib.ccfj_batch_graph_cache_clear()
        # the same work as 512 separate transforms
        single = []
        for b in range(nsets):
            o = int(off[b])
            n = int(counts[b])
            single.append(_dev_args(lib, torch, n, nf, nc, 1, 0, U.data_ptr(), 2 * nf, 2,
                                    perm.data_ptr() + 8 * o, r_sorted[o:o + n], f32, c32,
                                    out[b]))
            single[-1].u_rows = total

        def separate():
            for a in single:
                _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))

        t_sep = _time_device(separate, 1, 1)
        terms = total * nf * nc
        # FP64 station-amortised form of 8 subarrays (the largest, the
        # smallest and 6 in between) against the batch's FP32 output
        with torch.cuda.stream(s_cap):
            batch_step()
        s_cap.synchronize()
        y32 = out.cpu().numpy()
        lib.ccfj_batch_graph_cache_clear()
        picks = np.unique(np.argsort(counts)[np.linspace(0, nsets - 1, 8).astype(int)])
        o64 = torch.empty((nc, nf), device="cuda")
        errs = []
        for b in picks:
            a = single[b]
            a.precision, a.out = _lib.PREC_FP64, o64.data_ptr()
            _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))
            torch.cuda.synchronize()
            errs.append(_max_err(y32[b], o64.cpu().numpy(), "")["max_abs_err_vs_fp64_normalised"])
        res["accuracy"] = {"max_abs_err_vs_fp64_normalised": float(np.nanmax(errs)),
                           "sample": "subarrays with %s pairs" % ", ".join(str(int(counts[b]))
                                                                          for b in picks)}
        res.update(workload="%d subarrays, %d pairs in total (log-uniform 50-20000 each), "
                            "nf=1024, nc=500, itype=1 func=0; one persistent graph-replayed "
                            "launch" % (nsets, total), seconds=t_batch, value=terms / t_batch,
                   separate_launches_seconds=t_sep, separate_launches_value=terms / t_sep,
                   speedup_vs_separate=t_sep / t_batch)
    print(json.dumps(res))
    return 0


def _quiet(fn, *a, **k):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return fn(*a, **k)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--profile-case", nargs="?", const="noise", default=None,
                    choices=("noise", "hilbert", "mwfj", "mwfj_cc", "batch", "cc"),
                    help="run a reduced case for ncu captures: 'noise' = the device transform "
                         "on the first 512 frequencies of the workload (steps launches, no "
                         "extras); 'mwfj' = the MWFJ configuration with 8 windows and 256 bins; "
                         "'hilbert' = the same with func 1 (device Hilbert transform); 'mwfj_cc' "
                         "= the MWFJ case with func 1 (CUDA-core kernel); 'batch' = the ragged "
                         "batch with 64 subarrays; 'cc' = cross-correlation of the reference "
                         "example's day (one JSON line)")
    ap.add_argument("--config", type=int, default=0, choices=(0, 1, 3, 4, 5),
                    help="time another workload (device-resident; one JSON line): 1 small noise array, "
                         "3 earthquake, 4 MWFJ, 5 ragged batch")
    args = ap.parse_args()
    if args.config:
        return run_config(args)
    if args.profile_case in ("mwfj", "mwfj_cc"):
        args.config = 4
        args.mwfj_small = True
        args.mwfj_func = 1 if args.profile_case == "mwfj_cc" else 0
        return run_config(args)
    if args.profile_case == "cc":
        return run_cc_case(args)
    if args.profile_case == "batch":
        args.config = 5
        args.batch_small = True
        return run_config(args)
    if args.profile_case:
        return run_profile_case(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world)


if __name__ == "__main__":
    sys.exit(main())
