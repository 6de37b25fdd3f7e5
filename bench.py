#!/usr/bin/env python3
"""Benchmark of the B200 F-J transform on the five benchmark configurations.

Headline (one "step"): ccfj fj_noise, itype=1 (linear-interpolation
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

The same line carries a `configs` object with the other four workloads, each
with its device-resident value, its end-to-end value through the public API
on host arrays, a roofline figure, the reference's CPU rate on a sample of
the same workload, and its error against the FP64 GPU form (every cell), the
FP64 oracle and the reference's own FJcpu.cpp output (sampled columns):
  1  fj_noise, 200 pairs x 512 f x 300 c
  3  fj_earthquake with the device rFFT, 500 traces x 8192 samples, nf 1024,
     nc 800
  4  MWFJ, 1000 traces x 16384 samples, 64 windows, nf 1024, nc 2000
     (tensor cores)
  5  ragged batch, 512 subarrays (50-20,000 pairs each), nf 1024, nc 500, one
     persistent graph-replayed launch

  --impl reference   times the reference's own CPU implementation
          (src/ccfj.pyx over src/FJcpu.cpp with OpenMP, built into
          oracle/_ref by `make -C oracle`) on the headline workload: every
          step transforms one frequency column per host thread (FJcpu.cpp
          parallelises over frequencies), and the steps rotate through
          evenly spaced columns of the whole band.

Multi-GPU (torchrun): every rank transforms its own copy of the headline
workload (the transform shards by frequency or by data set with no exchange:
weak scaling); time is the max over ranks. The other configurations are
measured on rank 0 of single-GPU runs.
"""
import argparse
import ctypes
import json
import multiprocessing
import os
import statistics
import subprocess
import sys
import tempfile
import time
import warnings

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(REPO, "oracle"), os.path.join(REPO, "tests"),
           os.path.join(REPO, "cc-fjpy_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "F-J terms/s (nf·nc·npairs), FP32/batched vs FP64 GPU form at ≤1e-4 rel err"
NPAIRS, NF, NC = 19900, 2048, 1000
# Algorithmic FLOPs per (f, c, pair) term, FMA = 2, special-function unit
# operations not counted: a station evaluation E (J0 and J1 with a shared
# phase, the Struve remainder, the B(x) combine) and an interval combine A
# per real input.
FLOPS_E1, FLOPS_A1 = 104, 24     # itype 1
FLOPS_PER_TERM_ITYPE1 = FLOPS_E1 + FLOPS_A1
FALLBACK_BF16_TFLOPS = 1590.0


# ------------------------------------------------------------- workloads
def workload(seed=2):
    """The headline workload (configuration 2)."""
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


def workload_small(seed=1):
    """Configuration 1: 200 sorted pairs r ~ U(1, 50) km, 512 f over 0.01-1 Hz,
    300 c over 1000-5000 m/s, sigma = 0.1."""
    import cases
    rng = np.random.default_rng(seed)
    r = np.sort(rng.uniform(1e3, 5e4, 200))
    f = np.linspace(0.01, 1.0, 512)
    c = np.linspace(1000.0, 5000.0, 300)
    return cases.noise_spectra(rng, r, f, sigma=0.1), r, f, c


def workload_eq(seed=3):
    """Configuration 3: 500 dispersed Ricker traces of 8192 samples at 20 Hz,
    r log-uniform 10-2000 km, bins 0..1023, 800 c over 2000-5000 m/s."""
    import cases
    rng = np.random.default_rng(seed)
    ntr, npts, Fs, nf = 500, 8192, 20.0, 1024
    r = np.exp(rng.uniform(np.log(1e4), np.log(2e6), ntr))
    c = np.linspace(2000.0, 5000.0, 800)
    u = cases.ricker_records(rng, r, npts, Fs)
    f = Fs * np.arange(nf) / npts
    return u, r, f, c


def workload_mwfj(seed=4, nf=1024, nwin=64):
    """Configuration 4: 1000 traces of 16384 samples at 10 Hz, r log-uniform
    5-1500 km, 64 windows per trace (length 200-2000 samples at a uniform
    start, in seconds), taper 0.9, bins 0..1023, 2000 c over 1500-5000 m/s."""
    import cases
    rng = np.random.default_rng(seed)
    ntr, npts, Fs = 1000, 16384, 10.0
    r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e6), ntr))
    c = np.linspace(1500.0, 5000.0, 2000)
    u = cases.ricker_records(rng, r, npts, Fs)
    f = Fs * np.arange(nf) / npts
    L = rng.integers(200, 2001, size=(nwin, ntr))
    start = rng.integers(0, npts - L)
    return dict(u=u, r=r, f=f, c=c, Fs=Fs, nwin=nwin, winl=start / Fs, winr=(start + L) / Fs,
                taper=0.9)


def batch_counts(seed=5, nsets=512):
    """Configuration 5's subarray sizes: log-uniform 50-20,000 pairs."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(50), np.log(20000), nsets)).astype(np.int64)
    return counts, np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


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


def bf16_peak():
    """Dense bf16 tensor peak in TFLOP/s: the burst figure of
    MEASURED_PEAKS.json when present, else the pool's fallback."""
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        for k, v in d.items():
            if "bf16" in k and "sustained" not in k and isinstance(v, (int, float)):
                return float(v), "MEASURED_PEAKS.json %s (measured)" % k
    except (OSError, ValueError, AttributeError):
        pass
    return FALLBACK_BF16_TFLOPS, "fallback 1590 TFLOP/s (MEASURED_PEAKS.json absent)"


# ------------------------------------------------------------ CPU baseline
def reference_module():
    ref_dir = os.path.join(REPO, "oracle", "_ref")
    if ref_dir not in sys.path:
        sys.path.insert(0, ref_dir)
    import ccfj_ref  # the reference's Cython module over FJcpu.cpp
    return ccfj_ref


def host_threads():
    return os.cpu_count() or 1


def column_sets(nf, per_step, steps):
    """`steps` sets of `per_step` columns: together evenly spaced over all nf
    columns, each set itself spread over the band (set s = every steps-th
    column from offset s)."""
    allc = np.unique(np.linspace(0, nf - 1, per_step * steps).round().astype(int))
    return [allc[s::steps] for s in range(steps)]


def ref_noise_cols(ref, uf, r, c, f, cols, threads):
    """The reference's fj_noise on the frequency columns `cols` (every column
    is independent, normalisation included): (seconds, float32 [nc, ncols])."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        t0 = time.perf_counter()
        out = ref.fj_noise(uf[:, cols], r, c, f[cols], itype=1, func=0, num=threads)
        return time.perf_counter() - t0, out


def _normalize_builtin(out):
    with np.errstate(all="ignore"):
        for i in range(out.shape[1]):
            out[:, i] = out[:, i] / max(np.abs(out[:, i]))
    return out


def ref_eq_cols(ref, u, r, c, f, cols, threads):
    """The reference's fj_earthquake (src/ccfj.pyx:229-250) restricted to the
    bins `cols`: the same argsort and np.fft.rfft of every trace, then its
    own `fj` on the real and imaginary parts of those bins, the magnitude and
    the per-column normalisation. Returns (seconds of the rfft, seconds of
    the fj calls, float32 [nc, ncols])."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        t0 = time.perf_counter()
        indx = np.argsort(r)
        rs = r[indx]
        uf = np.fft.rfft(u[indx])
        t1 = time.perf_counter()
        ufr, ufi = np.real(uf[:, cols]), np.imag(uf[:, cols])
        fc = f[cols]
        outr = ref.fj(ufr, rs, c, fc, 1, 1, threads)
        outi = ref.fj(ufi, rs, c, fc, 1, 1, threads)
        out = np.sqrt(outr ** 2 + outi ** 2)
        t2 = time.perf_counter()
    return t1 - t0, t2 - t1, _normalize_builtin(out)


def ref_mwfj_window_cols(ref, wl, w, cols, threads):
    """One window of the reference's MWFJ (src/ccfj.pyx:252-268): its `win`
    taper per trace, then fj_earthquake on the bins `cols`. Returns (seconds
    of taper + rfft, seconds of the fj calls, float32 [nc, ncols])."""
    u, r = wl["u"], wl["r"]
    nr, npts = u.shape
    t0 = time.perf_counter()
    u0 = np.zeros([nr, npts])
    for j in range(nr):
        u0[j, :] = u[j, :] * ref.win(npts, wl["Fs"], wl["winl"][w, j], wl["winr"][w, j], wl["taper"])
    t_win = time.perf_counter() - t0
    t_fft, t_fj, out = ref_eq_cols(ref, u0, r, wl["c"], wl["f"], cols, threads)
    return t_win + t_fft, t_fj, out


def cpu_line(terms, seconds, threads, sample):
    return {"value": terms / seconds, "unit": "terms/s", "cores": threads, "kind": "reference",
            "sample": sample}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    uf, r, f, c = workload()
    threads = host_threads()
    try:
        ref = reference_module()
    except ImportError as e:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built: %s" % e}))
        return 0
    sets = column_sets(NF, threads, args.steps)
    warm = column_sets(NF, threads, max(args.warmup, 1))
    for k in range(args.warmup):
        ref_noise_cols(ref, uf, r, c, f, warm[k], threads)
    t = 0.0
    ncols = 0
    for cols in sets:
        t += ref_noise_cols(ref, uf, r, c, f, cols, threads)[0]
        ncols += len(cols)
    value = ncols * NC * NPAIRS / t
    sample = ("reference fj_noise (src/ccfj.pyx + src/FJcpu.cpp, OpenMP over frequencies, %d "
              "threads): %d columns per step (one per thread), the %d steps together %d evenly "
              "spaced of the %d frequencies; all %d pairs and %d velocities" %
              (threads, len(sets[0]), args.steps, ncols, NF, NPAIRS, NC))
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


# ----------------------------------------------------------------- oracle
def _oracle_job(job):
    """One FP64 oracle evaluation in a worker process (spawned, so it holds
    no CUDA state): returns float64 [nc, ncols]."""
    import fj_oracle as O
    kind, p = job
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        if kind == "noise":
            return O.fj_noise(p["uf"], p["r"], p["c"], p["f"])
        if kind == "eq":
            return O.fj_earthquake_columns(p["u"], p["r"], p["c"], p["f"], p["cols"])
        if kind == "mwfj":
            return O.mwfj_window_columns(p["u"], p["r"], p["c"], p["f"], p["Fs"], p["winl"],
                                         p["winr"], p["cols"], p["taper"])
    raise ValueError(kind)


def _err(y, ref):
    """max over the cells of |y - ref| / max_c |ref(:, f)| (the error of the
    normalised spectrum), over the columns where ref is finite."""
    import fj_oracle as O
    return O.rel_error(y, ref)


def _nan_equal(a, b):
    return bool(np.array_equal(np.isnan(a), np.isnan(b)))


# -------------------------------------------------------------- helpers
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


def _time_profiled(lib, fn, steps, warmup, dev):
    """Device time per call (CUDA events around the calls on the current
    stream), the library's own event time of its main kernel per call,
    launches per call and the clocks seen."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_smi_index(dev))
    lib.ccfj_profile_enable(1)
    l0 = lib.ccfj_launch_count()
    s = _time_device(fn, steps, 0)
    launches = (lib.ccfj_launch_count() - l0) / steps
    cnt = ctypes.c_int(0)
    kern = lib.ccfj_profile_total_ms(ctypes.byref(cnt))
    lib.ccfj_profile_enable(0)
    clocks = sampler.stop()
    return s, (kern / cnt.value / 1e3 if cnt.value else None), launches, clocks


def _time_host_calls(fn, steps, warmup):
    """Seconds per call of a host-memory API call (synchronous), timed with
    CUDA events on the current stream around the calls, with the result of
    the last call."""
    import torch
    out = None
    for _ in range(warmup):
        out = fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps, out


def _fj_args(nr, nf, nc, itype, mode, u_ptr, u_ld, u_es, perm_ptr, r_t, f_t, c_t, out_t,
             u2_ptr=None, hilbert=0, ncols=None, u_rows=None, precision=0):
    from ccfj import _lib
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nr, a.nf, a.nc = nr, nf, nc
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = itype, mode, precision, 1, 1
    a.hilbert = hilbert
    a.u[0] = u_ptr
    a.u[1] = u2_ptr
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = u_ld, u_rows or nr, u_es, ncols or nf, 1
    a.perm = perm_ptr or None
    a.r, a.f, a.c, a.out = r_t.data_ptr(), f_t.data_ptr(), c_t.data_ptr(), out_t.data_ptr()
    return a


def _fp32_roofline(flops, kernel_s, peak, kernel, flops_per_term, traffic=None):
    ach = flops / kernel_s / 1e12
    return {"bound": "fp32", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "traffic": traffic, "kernel": kernel, "kernel_ms": kernel_s * 1e3,
            "flops_per_term": flops_per_term,
            "peak_source": "FP32 FMA probe at bench time (ccfj_fp32_peak_probe), measured"}


def profile_traffic(name):
    """DRAM bytes per launch of a kernel from a committed ncu summary under
    profiles/ (the line 'traffic_bytes_per_launch: <bytes>'), or None."""
    p = os.path.join(REPO, "profiles", name)
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def traffic_per_launch():
    return profile_traffic("fj_amortized_config2.md")


# ------------------------------------------------------------ the configs
class ConfigRun:
    """One configuration: device measurements first (GPU), then the
    reference's CPU sample (all host threads, nothing else running), then
    the oracle jobs (a spawned process pool). Each stage fills `res`."""

    def __init__(self, cid):
        self.cid = cid
        self.res = {}
        self.gpu_cols = None      # float32 [.., nc, ncols] GPU output on the sampled columns
        self.y64_cols = None      # the FP64 GPU form on the same columns
        self.ref_out = None       # the reference's output on them
        self.oracle_jobs = []     # (job, slice of gpu_cols it covers)

    def finish(self, oracle_outs):
        acc = self.res.setdefault("accuracy", {})
        if self.ref_out is not None:
            acc["err_vs_fjcpu"] = _err(self.gpu_cols, self.ref_out)
            acc["fjcpu_err_vs_fp64"] = _err(self.ref_out, self.y64_cols)
            acc["nan_positions_equal_fjcpu"] = _nan_equal(self.gpu_cols, self.ref_out)
        if oracle_outs:
            eg, er = [], []
            for (job, sl), o in zip(self.oracle_jobs, oracle_outs):
                eg.append(_err(self.gpu_cols[sl], o))
                if self.ref_out is not None:
                    er.append(_err(self.ref_out[sl], o))
            acc["err_vs_oracle"] = float(max(eg))
            if er:
                acc["fjcpu_err_vs_oracle"] = float(max(er))
        if "err_vs_fjcpu" in acc:
            own = max(acc.get("fjcpu_err_vs_oracle", 0.0), acc["fjcpu_err_vs_fp64"])
            acc["fjcpu_check"] = ("err_vs_fjcpu %.2e <= FJcpu's own error %.2e + 1e-4: %s" %
                                  (acc["err_vs_fjcpu"], own, acc["err_vs_fjcpu"] <= own + 1e-4))
        return self.res


def measure_small(lib, torch, dev, sp, peak, args):
    """Configuration 1 on the device and end to end."""
    import ccfj
    from ccfj import _lib
    run = ConfigRun(1)
    uf, r, f, c = workload_small()
    nr, nf, nc = len(r), len(f), len(c)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=uf.view(np.float32), r=r.astype(np.float32), f=f.astype(np.float32),
        c=c.astype(np.float32)).items()}
    out = torch.empty((nc, nf), device="cuda")
    a = _fj_args(nr, nf, nc, 1, _lib.MODE_J, d["u"].data_ptr(), 2 * nf, 2, None, d["r"], d["f"],
                 d["c"], out)
    fn = lambda: _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))  # noqa: E731
    # the tile choice (velocities per thread x station ranges) from the
    # project's autotuner, recorded for this problem class before timing
    best, best_ms = ctypes.c_int(), ctypes.c_float()
    _lib.check(lib.ccfj_autotune_fj_v1(ctypes.byref(a), sp, ctypes.byref(best),
                                       ctypes.byref(best_ms)))
    cpt, nsplit = ctypes.c_int(), ctypes.c_int()
    _lib.check(lib.ccfj_tuned_choice_fj(ctypes.byref(a), ctypes.byref(cpt), ctypes.byref(nsplit)))
    s, ks, launches, clocks = _time_profiled(lib, fn, 200, 10, dev)
    y32 = out.cpu().numpy()
    a.precision = _lib.PREC_FP64
    fn()
    y64 = out.cpu().numpy()
    terms = nr * nf * nc
    te, ye = _time_host_calls(lambda: _quiet(ccfj.fj_noise, uf, r, c, f), 20, 3)
    run.res = {
        "workload": "fj_noise itype=1 func=0: 200 sorted pairs (1-50 km) x 512 f (0.01-1 Hz) x "
                    "300 c (1000-5000 m/s), sigma 0.1", "unit": "terms/s",
        "value": terms / s, "ms_per_call": s * 1e3, "gpu_launches_per_call": launches,
        "clocks": clocks,
        "tile_choice": {"velocities_per_thread": cpt.value, "station_ranges": nsplit.value,
                        "source": "ccfj_autotune_fj_v1 (best of 1/2/4 velocities per thread x "
                                  "1-8 station ranges, %.3f ms)" % best_ms.value},
        "e2e": {"value": terms / te, "unit": "terms/s", "ms_per_call": te * 1e3,
                "h2d_bytes_per_step": int(uf.nbytes + r.nbytes + 8 * nr + 4 * (nf + nc)),
                "d2h_bytes_per_step": int(ye.nbytes)},
        "roofline": _fp32_roofline(FLOPS_PER_TERM_ITYPE1 * terms, ks, peak,
                                   "fj_amortized_kernel<MODE_J, 1, float, %d>" % cpt.value,
                                   FLOPS_PER_TERM_ITYPE1,
                                   traffic=profile_traffic("fj_split_small_array.md")),
        "accuracy": {"max_abs_err_vs_fp64_normalised": _err(y32, y64),
                     "nan_positions_equal_fp64": _nan_equal(y32, y64),
                     "fp64_sample": "all 300 x 512 cells", "e2e_equals_device": bool(
                         np.array_equal(ye, y32, equal_nan=True))},
    }
    run.uf, run.r, run.f, run.c = uf, r, f, c
    run.gpu_cols, run.y64_cols = y32, y64
    return run


def cpu_small(run, ref, threads):
    t = 0.0
    out = None
    for _ in range(2):
        dt, out = ref_noise_cols(ref, run.uf, run.r, run.c, run.f, np.arange(len(run.f)), threads)
        t += dt
    terms = 2 * run.uf.shape[0] * len(run.f) * len(run.c)
    run.res["cpu_baseline"] = cpu_line(terms, t, threads,
                                       "reference fj_noise on the whole workload, 2 calls (%.1f s)"
                                       % t)
    run.ref_out = out
    run.res["accuracy"]["fjcpu_sample"] = "all 300 x 512 cells"
    cols = np.array_split(np.arange(len(run.f)), 16)
    run.oracle_jobs = [(("noise", dict(uf=run.uf[:, cc], r=run.r, c=run.c, f=run.f[cc])),
                        (slice(None), cc)) for cc in cols]
    run.res["accuracy"]["oracle_sample"] = "all 300 x 512 cells"


def measure_eq(lib, torch, dev, sp, peak, args):
    """Configuration 3 (fj_earthquake with the device rFFT)."""
    import ccfj
    from ccfj import _lib, _eq
    run = ConfigRun(3)
    u, r, f, c = workload_eq()
    ntr, npts = u.shape
    nf, nc = len(f), len(c)
    idx = np.argsort(r)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=u, perm=idx.astype(np.int64), r=r[idx].astype(np.float32), f=f.astype(np.float32),
        c=c.astype(np.float32)).items()}
    out = torch.empty((nc, nf), device="cuda")
    a = _eq.EqArgs()
    a.struct_size = ctypes.sizeof(a)
    a.ntr, a.npts, a.nf, a.nc = ntr, npts, nf, nc
    a.itype, a.func, a.precision, a.normalize, a.device_ptrs, a.fstride = 1, 0, 0, 1, 1, 1
    a.u, a.u_ld, a.u_rows = d["u"].data_ptr(), npts, ntr
    a.perm, a.r, a.f, a.c = (d[k].data_ptr() for k in ("perm", "r", "f", "c"))
    a.out = out.data_ptr()
    fn = lambda: _lib.check(lib.ccfj_fj_earthquake_v1(ctypes.byref(a), sp))  # noqa: E731
    s, ks, launches, clocks = _time_profiled(lib, fn, 20, 3, dev)
    y32 = out.cpu().numpy()
    a.precision = _lib.PREC_FP64
    fn()
    y64 = out.cpu().numpy()
    terms = ntr * nf * nc
    te, ye = _time_host_calls(lambda: _quiet(ccfj.fj_earthquake, u, r, c, f), 5, 2)
    fpt = FLOPS_E1 + 2 * FLOPS_A1
    run.res = {
        "workload": "fj_earthquake itype=1 func=0 with the device rFFT: 500 traces x 8192 "
                    "samples at 20 Hz (r 10-2000 km), bins 0-1023, nc=800 (2000-5000 m/s)",
        "unit": "terms/s", "value": terms / s, "ms_per_call": s * 1e3,
        "gpu_launches_per_call": launches, "clocks": clocks,
        "e2e": {"value": terms / te, "unit": "terms/s", "ms_per_call": te * 1e3,
                "h2d_bytes_per_step": int(u.nbytes + 4 * ntr + 8 * ntr + 4 * (nf + nc)),
                "d2h_bytes_per_step": int(ye.nbytes)},
        "roofline": _fp32_roofline(fpt * terms, ks, peak,
                                   "fj_amortized_kernel<MODE_ABS_J, 1, float, 2> (Re and Im "
                                   "share each station evaluation)", fpt),
        "accuracy": {"max_abs_err_vs_fp64_normalised": _err(y32, y64),
                     "nan_positions_equal_fp64": _nan_equal(y32, y64),
                     "fp64_sample": "all 800 x 1024 cells (the f = 0 column is NaN in every "
                                    "form, as in the reference)",
                     "e2e_equals_device": bool(np.array_equal(ye, y32, equal_nan=True))},
    }
    run.u, run.r, run.f, run.c = u, r, f, c
    run.y32_full, run.y64_full = y32, y64
    return run


def cpu_eq(run, ref, threads):
    nf = len(run.f)
    sets = column_sets(nf, threads, 2)
    sets[0] = np.unique(np.concatenate([[0], sets[0]]))  # bin 0: the NaN column
    t_fft = t_fj = 0.0
    outs, cols = [], []
    for cc in sets:
        a, b, o = ref_eq_cols(ref, run.u, run.r, run.c, run.f, cc, threads)
        t_fft += a
        t_fj += b
        outs.append(o)
        cols.append(cc)
    cols = np.concatenate(cols)
    # rate of the whole call: the rfft once per call, the fj time per column
    t = t_fj + t_fft / len(sets) * len(cols) / nf
    terms = len(cols) * run.u.shape[0] * len(run.c)
    run.res["cpu_baseline"] = cpu_line(
        terms, t, threads, "reference fj_earthquake steps (argsort, np.fft.rfft, its fj on Re and "
        "Im) on %d of %d bins (2 calls of one bin per thread, bin 0 included); the rfft's time is "
        "counted per bin (%.2f s of fj, %.2f s of rfft per call)" % (len(cols), nf, t_fj,
                                                                      t_fft / len(sets)))
    run.ref_out = np.concatenate(outs, axis=1)
    run.gpu_cols = run.y32_full[:, cols]
    run.y64_cols = run.y64_full[:, cols]
    run.res["accuracy"]["fjcpu_sample"] = "%d bins of all 800 velocities" % len(cols)
    pick = np.linspace(1, len(cols) - 1, 4).round().astype(int)
    run.oracle_jobs = [(("eq", dict(u=run.u, r=run.r, c=run.c, f=run.f, cols=cols[[k]])),
                        (slice(None), [k])) for k in pick]
    run.res["accuracy"]["oracle_sample"] = "bins %s" % cols[pick].tolist()


def measure_mwfj(lib, torch, dev, sp, peak, bf16, args):
    """Configuration 4 (MWFJ, 64 windows, tensor cores)."""
    import ccfj
    from ccfj import _lib, _eq
    run = ConfigRun(4)
    wl = workload_mwfj()
    u, r, f, c = wl["u"], wl["r"], wl["f"], wl["c"]
    ntr, npts = u.shape
    nf, nc, nwin = len(f), len(c), wl["nwin"]
    idx = np.argsort(r)
    n1, n2, dl = _eq._win_params(npts, wl["Fs"], wl["winl"], wl["winr"], wl["taper"])
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=u, perm=idx.astype(np.int64), r=r[idx].astype(np.float32), f=f.astype(np.float32),
        c=c.astype(np.float32), n1=n1.astype(np.int32), n2=n2.astype(np.int32),
        dl=dl.astype(np.int32)).items()}
    out = torch.empty((nwin, nc, nf), device="cuda")
    a = _eq.EqArgs()
    a.struct_size = ctypes.sizeof(a)
    a.ntr, a.npts, a.nf, a.nc, a.nwin = ntr, npts, nf, nc, nwin
    a.itype, a.func, a.precision, a.normalize, a.device_ptrs, a.fstride = 1, 0, 0, 1, 1, 1
    a.u, a.u_ld, a.u_rows = d["u"].data_ptr(), npts, ntr
    a.perm, a.r, a.f, a.c = (d[k].data_ptr() for k in ("perm", "r", "f", "c"))
    a.win_n1, a.win_n2, a.win_delta = (d[k].data_ptr() for k in ("n1", "n2", "dl"))
    a.out = out.data_ptr()
    fn = lambda: _lib.check(lib.ccfj_fj_earthquake_v1(ctypes.byref(a), sp))  # noqa: E731
    s, ks, launches, clocks = _time_profiled(lib, fn, 10, 2, dev)
    y32 = out.cpu().numpy()
    # FP64 station-amortised form of every window (one transform per window)
    a.precision = _lib.PREC_FP64
    t0 = time.perf_counter()
    fn()
    torch.cuda.synchronize()
    t64 = time.perf_counter() - t0
    y64 = out.cpu().numpy()
    terms = nwin * ntr * nf * nc
    te, ye = _time_host_calls(lambda: _quiet(ccfj.MWFJ, u, r, c, f, wl["Fs"], nwin, wl["winl"],
                                             wl["winr"], wl["taper"]), 3, 1)
    # tensor work: per frequency a (nc x K) (K x 2 nwin) product, K = 2 (ntr - 1),
    # in three fp16 passes (hi.hi + hi.lo + lo.hi)
    gemm = 2.0 * nc * (2 * nwin) * (2 * (ntr - 1)) * nf
    tc_ach = 3 * gemm / ks / 1e12
    gen = FLOPS_E1 * float(ntr) * nf * nc
    rl = _fp32_roofline(gen, ks, peak, "fj_mw_tc_kernel (A-operand generation on the FP32 pipe, "
                        "tcgen05 FP16x3 contraction)", FLOPS_E1)
    rl["flops_note"] = ("FP32 figure: the station evaluations E = 104 flops per (f, c, pair), "
                        "shared by all windows")
    rl["tensor"] = {"achieved": tc_ach, "peak": bf16[0], "unit": "TFLOP/s", "frac": tc_ach / bf16[0],
                    "peak_source": bf16[1], "flops": 3 * gemm,
                    "note": "2 nc (2 nwin) 2 (ntr - 1) nf algorithmic flops, x3 for the hi/lo split (FP16x3); the dense fp16 and bf16 peaks are equal"}
    run.res = {
        "workload": "MWFJ itype=1 func=0: 1000 traces x 16384 samples at 10 Hz (r 5-1500 km), "
                    "64 windows per trace (200-2000 samples, taper 0.9), bins 0-1023, nc=2000 "
                    "(1500-5000 m/s)", "unit": "window terms/s (nwin nf nc ntr)",
        "value": terms / s, "ms_per_call": s * 1e3, "gpu_launches_per_call": launches,
        "clocks": clocks,
        "e2e": {"value": terms / te, "unit": "window terms/s", "ms_per_call": te * 1e3,
                "h2d_bytes_per_step": int(u.nbytes + 12 * n1.size + 12 * ntr + 4 * (nf + nc)),
                "d2h_bytes_per_step": int(4 * nwin * nc * nf),
                "note": "MWFJ returns float64 (the reference's dtype): the library copies the "
                        "float32 result out through pinned staging on several host threads and "
                        "converts it to float64 on the way, inside the timed region"},
        "roofline": rl,
        "accuracy": {"max_abs_err_vs_fp64_normalised": _err(y32, y64),
                     "nan_positions_equal_fp64": _nan_equal(y32, y64),
                     "fp64_sample": "all 64 windows x 2000 x 1024 cells (FP64 form: %.1f s)" % t64,
                     "e2e_equals_device": bool(np.array_equal(ye.astype(np.float32), y32,
                                                               equal_nan=True))},
    }
    run.wl = wl
    run.y32_full, run.y64_full = y32, y64
    return run


def cpu_mwfj(run, ref, threads):
    wl = run.wl
    nf = len(wl["f"])
    wins = [5, 40]
    sets = column_sets(nf, threads, len(wins))
    t_pre = t_fj = 0.0
    outs, gpu, y64, ncols = [], [], [], 0
    for w, cc in zip(wins, sets):
        a, b, o = ref_mwfj_window_cols(ref, wl, w, cc, threads)
        t_pre += a
        t_fj += b
        outs.append(o)
        gpu.append(run.y32_full[w][:, cc])
        y64.append(run.y64_full[w][:, cc])
        ncols += len(cc)
    t = t_fj + t_pre * ncols / (nf * len(wins))
    terms = ncols * wl["u"].shape[0] * len(wl["c"])
    run.res["cpu_baseline"] = cpu_line(
        terms, t, threads, "reference MWFJ steps (win per trace, np.fft.rfft, its fj on Re and Im) "
        "for windows %s on %d bins each (one per thread); the taper and rfft time counted per bin "
        "(%.2f s of fj, %.2f s of taper+rfft per window)" % (wins, len(sets[0]), t_fj,
                                                            t_pre / len(wins)))
    run.ref_out = np.concatenate(outs, axis=1)
    run.gpu_cols = np.concatenate(gpu, axis=1)
    run.y64_cols = np.concatenate(y64, axis=1)
    run.res["accuracy"]["fjcpu_sample"] = "windows %s, %d bins each" % (wins, len(sets[0]))
    jobs = []
    off = 0
    for w, cc in zip(wins, sets):
        for k in (1, len(cc) - 1):
            jobs.append((("mwfj", dict(u=wl["u"], r=wl["r"], c=wl["c"], f=wl["f"], Fs=wl["Fs"],
                                       winl=wl["winl"][w], winr=wl["winr"][w], cols=cc[[k]],
                                       taper=wl["taper"])), (slice(None), [off + k])))
        off += len(cc)
    run.oracle_jobs = jobs
    run.res["accuracy"]["oracle_sample"] = "windows %s, 2 bins each" % wins


def measure_batch(lib, torch, dev, sp, peak, args):
    """Configuration 5 (ragged batch, one persistent graph-replayed launch)."""
    import ccfj
    from ccfj import _lib, _batch
    run = ConfigRun(5)
    nsets = 64 if getattr(args, "batch_small", False) else 512
    counts, off = batch_counts(nsets=nsets)
    total = int(off[-1])
    nf, nc = 1024, 500
    f = np.linspace(0.01, 1.0, nf)
    c = np.linspace(1000.0, 5000.0, nc)
    # spectra generated on the device (14 GB as complex64): the c(f) law with
    # an overtone and sigma = 0.2 noise, as the large-array workload
    g = torch.Generator(device="cuda").manual_seed(5)
    r_t = torch.rand(total, generator=g, device="cuda", dtype=torch.float64) * 299.5e3 + 500.0
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
    r_host = r_t.cpu().numpy()
    perm_h = np.concatenate([off[b] + np.argsort(r_host[off[b]:off[b + 1]])
                             for b in range(nsets)]).astype(np.int64)
    perm = torch.from_numpy(perm_h).cuda()
    r_sorted = torch.from_numpy(r_host[perm_h].astype(np.float32)).cuda()
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
    ba.perm, ba.f, ba.c, ba.out = perm.data_ptr(), f32.data_ptr(), c32.data_ptr(), out.data_ptr()
    s_cap = torch.cuda.Stream()
    spc = ctypes.c_void_p(s_cap.cuda_stream)
    fn = lambda: _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(ba), spc))  # noqa: E731
    with torch.cuda.stream(s_cap):
        s, _, launches, clocks = _time_profiled(lib, fn, 3, 1, dev)
    s_cap.synchronize()
    y32 = out.cpu().numpy()
    lib.ccfj_batch_graph_cache_clear()
    # the same work as separate plain launches, and the FP64 form of every subarray
    single = []
    for b in range(nsets):
        o = int(off[b])
        n = int(counts[b])
        a = _fj_args(n, nf, nc, 1, 0, U.data_ptr(), 2 * nf, 2, perm.data_ptr() + 8 * o,
                     r_sorted[o:o + n], f32, c32, out[b], u_rows=total)
        single.append(a)

    def separate():
        for a in single:
            _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))

    t_sep = _time_device(separate, 1, 1)
    o64 = torch.empty((nc, nf), device="cuda")
    errs = []
    nan_ok = True
    # the subarrays the CPU sample covers (stratified by size); their FP64
    # form is kept to compare FJcpu.cpp with on the same columns
    picks = np.argsort(counts)[np.linspace(0, nsets - 1, 8).round().astype(int)]
    y64_picked = {}
    t0 = time.perf_counter()
    for b in range(nsets):
        a = single[b]
        a.precision, a.out = _lib.PREC_FP64, o64.data_ptr()
        _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))
        y64b = o64.cpu().numpy()
        errs.append(_err(y32[b], y64b))
        nan_ok &= _nan_equal(y32[b], y64b)
        if b in picks:
            y64_picked[int(b)] = y64b
    t64 = time.perf_counter() - t0
    terms = total * nf * nc
    # end to end: host spectra in pinned memory, one view per subarray
    U_host = torch.empty((total, 2 * nf), dtype=torch.float32, pin_memory=True)
    U_host.copy_(U)
    Uc = U_host.numpy().view(np.complex64)
    ufs = [Uc[off[b]:off[b + 1]] for b in range(nsets)]
    rs = [r_host[off[b]:off[b + 1]] for b in range(nsets)]
    te, ye = _time_host_calls(lambda: _quiet(ccfj.fj_noise_batch, ufs, rs, c, f), 2, 1)
    e2e_eq = bool(all(np.array_equal(ye[b], y32[b], equal_nan=True) for b in range(nsets)))
    run.res = {
        "workload": "%d subarrays, %d pairs in total (log-uniform 50-20000 each, r 0.5-300 km), "
                    "nf=1024 (0.01-1 Hz), nc=500 (1000-5000 m/s), itype=1 func=0; one "
                    "persistent graph-replayed launch" % (nsets, total),
        "unit": "terms/s", "value": terms / s, "ms_per_call": s * 1e3,
        "gpu_launches_per_call": launches, "clocks": clocks,
        "separate_launches_ms": t_sep * 1e3, "speedup_vs_separate_launches": t_sep / s,
        "e2e": {"value": terms / te, "unit": "terms/s", "ms_per_call": te * 1e3,
                "h2d_bytes_per_step": int(U_host.numel() * 4 + 16 * total + 8 * (nsets + 1)
                                          + 4 * (nf + nc)),
                "d2h_bytes_per_step": int(4 * nsets * nc * nf),
                "note": "spectra in pinned host memory, one view per subarray"},
        "roofline": _fp32_roofline(FLOPS_PER_TERM_ITYPE1 * terms, s, peak,
                                   "fj_batch_persistent_kernel<MODE_J, 1, 2> (time of the whole "
                                   "graph replay)", FLOPS_PER_TERM_ITYPE1),
        "accuracy": {"max_abs_err_vs_fp64_normalised": float(max(errs)),
                     "nan_positions_equal_fp64": bool(nan_ok),
                     "fp64_sample": "all %d subarrays, every cell (FP64 form: %.1f s)" % (nsets,
                                                                                        t64),
                     "e2e_equals_device": e2e_eq},
    }
    # host copies of the subarrays the CPU sample covers
    run.sub = []
    for b in picks:
        ufb = Uc[off[b]:off[b + 1]].copy()
        run.sub.append((int(b), ufb, r_host[off[b]:off[b + 1]].copy(), y32[b],
                        y64_picked[int(b)]))
    run.f, run.c = f, c
    del U_host, Uc, ufs
    lib.ccfj_batch_graph_cache_clear()
    return run


def cpu_batch(run, ref, threads):
    nf = len(run.f)
    cols = column_sets(nf, threads, 1)[0]
    t = 0.0
    terms = 0
    outs, gpu, y64 = [], [], []
    for b, ufb, rb, y32b, y64b in run.sub:
        dt, o = ref_noise_cols(ref, ufb, rb, run.c, run.f, cols, threads)
        t += dt
        terms += len(rb) * len(cols) * len(run.c)
        outs.append(o)
        gpu.append(y32b[:, cols])
        y64.append(y64b[:, cols])
    run.res["cpu_baseline"] = cpu_line(
        terms, t, threads, "reference fj_noise on 8 subarrays stratified by size (%s pairs), %d "
        "evenly spaced of %d frequencies each (one per thread)" % (
            ",".join(str(len(x[2])) for x in run.sub), len(cols), nf))
    run.ref_out = np.concatenate(outs, axis=1)
    run.gpu_cols = np.concatenate(gpu, axis=1)
    run.y64_cols = np.concatenate(y64, axis=1)
    run.res["accuracy"]["fjcpu_sample"] = "8 subarrays x %d frequencies" % len(cols)
    jobs = []
    mid = len(cols) // 2
    for k in range(0, len(run.sub), 2):
        b, ufb, rb = run.sub[k][:3]
        jobs.append((("noise", dict(uf=ufb[:, cols[[mid]]], r=rb, c=run.c, f=run.f[cols[[mid]]])),
                     (slice(None), [k * len(cols) + mid])))
    run.oracle_jobs = jobs
    run.res["accuracy"]["oracle_sample"] = "4 subarrays x 1 frequency"


def finish_batch(run, oracle_outs):
    acc = run.res["accuracy"]
    acc["err_vs_fjcpu"] = _err(run.gpu_cols, run.ref_out)
    acc["nan_positions_equal_fjcpu"] = _nan_equal(run.gpu_cols, run.ref_out)
    eg, er = [], []
    for (job, sl), o in zip(run.oracle_jobs, oracle_outs):
        eg.append(_err(run.gpu_cols[sl], o))
        er.append(_err(run.ref_out[sl], o))
    acc["err_vs_oracle"] = float(max(eg))
    acc["fjcpu_err_vs_oracle"] = float(max(er))
    # FJcpu's own error on the columns it was compared on (against the FP64
    # form, which the oracle pins), and on the oracle's columns
    acc["fjcpu_err_vs_fp64"] = _err(run.ref_out, run.y64_cols)
    own = max(acc["fjcpu_err_vs_oracle"], acc["fjcpu_err_vs_fp64"])
    acc["fjcpu_check"] = ("err_vs_fjcpu %.2e <= FJcpu's own error %.2e + 1e-4: %s" %
                          (acc["err_vs_fjcpu"], own, acc["err_vs_fjcpu"] <= own + 1e-4))
    return run.res


# -------------------------------------------------------------- our arm
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

    def args_for(prec, nf=NF, out=d_out, u=d_u, fv=d_f, ld=2 * NF):
        a = _lib.FjArgs()
        a.struct_size = ctypes.sizeof(a)
        a.nr, a.nf, a.nc = NPAIRS, nf, NC
        a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, _lib.MODE_J, prec, 1, 1
        a.u[0] = u.data_ptr()
        a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = ld, NPAIRS, 2, nf, 1
        a.perm = d_perm.data_ptr()
        a.r, a.f, a.c, a.out = d_r.data_ptr(), fv.data_ptr(), d_c.data_ptr(), out.data_ptr()
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
        dist.barrier()
        dist.destroy_process_group()
    e2e = {"value": world * terms * e2e_steps / t_e2e, "unit": "terms/s",
           "h2d_bytes_per_step": int(uf.nbytes + rs.nbytes + idx.astype(np.int64).nbytes
                                     + 4 * (NF + NC)),
           "d2h_bytes_per_step": int(ccfj_out.nbytes), "wall_s_per_step": wall / e2e_steps}
    if rank != 0:
        return 0

    # ---- rank 0: accuracy, comparators, the other configurations (after the
    # process group is gone: the other ranks do not wait on this)
    y32 = d_out.cpu().numpy()
    d64 = torch.empty_like(d_out)
    _lib.check(lib.ccfj_fj_v1(ctypes.byref(args_for(_lib.PREC_FP64, out=d64)), sp))
    torch.cuda.synchronize()
    y64 = d64.cpu().numpy()
    err = _err(y32, y64)
    # the plain FP64 form (the reference's loop structure) on 64 evenly
    # spaced frequencies, after a warm-up launch, best of 3
    pcols = np.linspace(0, NF - 1, 64).round().astype(int)
    d_usub = d_u.view(NPAIRS, NF, 2)[:, torch.from_numpy(pcols).cuda(), :].contiguous()
    d_fsub = d_f[torch.from_numpy(pcols).cuda()].contiguous()
    d_pl = torch.empty((NC, len(pcols)), dtype=torch.float32, device="cuda")
    apl = args_for(_lib.PREC_FP64_PLAIN, nf=len(pcols), out=d_pl, u=d_usub, fv=d_fsub,
                   ld=2 * len(pcols))
    plain_s = min(_time_device(lambda: _lib.check(lib.ccfj_fj_v1(ctypes.byref(apl), sp)), 1, 1)
                  for _ in range(3))
    plain_tps = len(pcols) * NC * NPAIRS / plain_s
    apl32 = args_for(_lib.PREC_FP32, nf=len(pcols), out=d_pl, u=d_usub, fv=d_fsub,
                     ld=2 * len(pcols))
    sub32_s = min(_time_device(lambda: _lib.check(lib.ccfj_fj_v1(ctypes.byref(apl32), sp)), 1, 1)
                  for _ in range(3))
    peak = ctypes.c_double(0)
    _lib.check(lib.ccfj_fp32_peak_probe(sp, ctypes.byref(peak)))
    peak = peak.value
    achieved = FLOPS_PER_TERM_ITYPE1 * terms / (kern_ms / 1e3) / 1e12
    bf16 = bf16_peak()

    runs = []
    if world > 1:
        # scaling runs report the headline only: the other configurations and
        # the CPU baseline are single-GPU measurements (rank 0 at N = 1)
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "terms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; spectra from the c(f) dispersion law)",
            "config": config_dict(), "e2e": e2e, "clocks": clocks, "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic_per_launch(),
                         "kernel": "fj_amortized_kernel<MODE_J, itype 1, float>",
                         "kernel_ms": kern_ms, "flops_per_term": FLOPS_PER_TERM_ITYPE1},
            "accuracy": {"max_abs_err_vs_fp64_normalised": err}}))
        return 0
    if not args.headline_only:
        for meas in (measure_small, measure_eq):
            runs.append(meas(lib, torch, dev, sp, peak, args))
        runs.append(measure_mwfj(lib, torch, dev, sp, peak, bf16, args))
        runs.append(measure_batch(lib, torch, dev, sp, peak, args))

    # ---- CPU: the reference on every sample (all host threads, nothing else running)
    threads = host_threads()
    head = {}
    try:
        ref = reference_module()
    except ImportError as e:
        ref = None
        cpu = {"unavailable": "oracle/_ref not built: %s" % e}
    oracle_jobs, finishers = [], []
    if ref is not None:
        sets = column_sets(NF, threads, 2)
        tsum, outs = 0.0, []
        for cc in sets:
            dt, o = ref_noise_cols(ref, uf, r, c, f, cc, threads)
            tsum += dt
            outs.append(o)
        hcols = np.concatenate(sets)
        cpu = cpu_line(len(hcols) * NC * NPAIRS, tsum, threads,
                       "reference fj_noise (src/ccfj.pyx + src/FJcpu.cpp, OpenMP over frequencies, "
                       "%d threads): 2 calls of %d columns (one per thread), together %d evenly "
                       "spaced of the %d frequencies; all %d pairs and %d velocities (%.1f s)" %
                       (threads, len(sets[0]), len(hcols), NF, NPAIRS, NC, tsum))
        head_ref = np.concatenate(outs, axis=1)
        head["err_vs_fjcpu"] = _err(y32[:, hcols], head_ref)
        head["fjcpu_err_vs_fp64"] = _err(head_ref, y64[:, hcols])
        head["fjcpu_sample"] = "%d evenly spaced frequencies x all 1000 velocities" % len(hcols)
        opick = np.linspace(0, len(hcols) - 1, 4).round().astype(int)
        head_jobs = [("noise", dict(uf=uf[:, hcols[[k]]], r=r, c=c, f=f[hcols[[k]]]))
                     for k in opick]
        head["oracle_sample"] = "frequencies %s Hz x all 1000 velocities" % [
            round(float(f[hcols[k]]), 4) for k in opick]
        for run, cpu_fn in zip(runs, (cpu_small, cpu_eq, cpu_mwfj, cpu_batch)):
            cpu_fn(run, ref, threads)
        oracle_jobs = head_jobs + [j for run in runs for j, _ in run.oracle_jobs]

    # ---- oracle: spawned workers (no CUDA state), after the CPU timing
    oracle_outs = []
    if oracle_jobs:
        ctx = multiprocessing.get_context("spawn")
        with ctx.Pool(min(len(oracle_jobs), threads)) as pool:
            oracle_outs = pool.map(_oracle_job, oracle_jobs, chunksize=1)
    if ref is not None:
        ho = oracle_outs[:len(head_jobs)]
        head["err_vs_oracle"] = float(max(_err(y32[:, hcols[[k]]], o) for k, o in zip(opick, ho)))
        head["fjcpu_err_vs_oracle"] = float(max(_err(head_ref[:, [k]], o)
                                                for k, o in zip(opick, ho)))
        own = max(head["fjcpu_err_vs_oracle"], head["fjcpu_err_vs_fp64"])
        head["fjcpu_check"] = ("err_vs_fjcpu %.2e <= FJcpu's own error %.2e + 1e-4: %s" %
                               (head["err_vs_fjcpu"], own, head["err_vs_fjcpu"] <= own + 1e-4))
        pos = len(head_jobs)
        for run in runs:
            n = len(run.oracle_jobs)
            outs = oracle_outs[pos:pos + n]
            pos += n
            finishers.append(finish_batch(run, outs) if run.cid == 5 else run.finish(outs))
    else:
        finishers = [run.res for run in runs]

    result = {
        "metric": METRIC, "value": value, "unit": "terms/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; spectra from the c(f) dispersion law)",
        "config": config_dict(), "e2e": e2e,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic_per_launch(),
                     "kernel": "fj_amortized_kernel<MODE_J, itype 1, float>",
                     "kernel_ms": kern_ms,
                     "flops_per_term": FLOPS_PER_TERM_ITYPE1,
                     "peak_source": "measured at bench time: FP32 FMA probe "
                                    "(ccfj_fp32_peak_probe); MEASURED_PEAKS.json has no FP32 "
                                    "figure"},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": int(launches),
        "accuracy": dict({"max_abs_err_vs_fp64_normalised": err,
                          "fp64_sample": "all 1000 x 2048 cells",
                          "fp64_plain_terms_per_s": plain_tps,
                          "speedup_vs_fp64_plain": value / world / plain_tps,
                          "speedup_sample": "the plain FP64 form on 64 evenly spaced frequencies "
                                            "(0.005-2 Hz), warm, best of 3 launches: %.1f ms; the "
                                            "FP32 form on the same 64 columns: %.1f ms (%.1fx)" % (
                                                plain_s * 1e3, sub32_s * 1e3,
                                                plain_s / sub32_s)}, **head),
        "configs": {str(run.cid): res for run, res in zip(runs, finishers)},
    }
    print(json.dumps(result))
    return 0


def run_profile_extra(args):
    """Reduced cases for ncu captures of the kernels the main workloads do
    not launch: 'noise0' = the trapezoid (itype 0) transform of the first 512
    frequencies of the large-array workload; 'eq_short' = fj_earthquake on
    500 traces of 512 samples (radix-2 FFT) and of 3000 samples (direct
    DFT), 200 bins, 400 velocities; 'small' = the small-array workload
    (split launch over station ranges); 'cc_direct' = cross-correlation of
    50 stations x 86,400 samples in windows of 3001 samples (direct
    transform of the requested bins)."""
    import torch
    import ccfj
    from ccfj import _lib
    lib = _lib.load()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = args.warmup + args.steps
    if args.profile_case == "noise0":
        uf, r, f, c = workload()
        nf = 512
        idx = np.argsort(r)
        T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
            u=uf.view(np.float32), perm=idx.astype(np.int64), r=r[idx].astype(np.float32),
            f=f.astype(np.float32), c=c.astype(np.float32)).items()}
        out = torch.empty((NC, nf), device="cuda")
        a = _fj_args(NPAIRS, nf, NC, 0, _lib.MODE_J, T["u"].data_ptr(), 2 * NF, 2,
                     T["perm"].data_ptr(), T["r"], T["f"], T["c"], out)
        for _ in range(n):
            _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))
    elif args.profile_case == "small":
        uf, r, f, c = workload_small()
        T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
            u=uf.view(np.float32), r=r.astype(np.float32), f=f.astype(np.float32),
            c=c.astype(np.float32)).items()}
        out = torch.empty((len(c), len(f)), device="cuda")
        a = _fj_args(len(r), len(f), len(c), 1, _lib.MODE_J, T["u"].data_ptr(), 2 * len(f), 2,
                     None, T["r"], T["f"], T["c"], out)
        for _ in range(n):
            _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), sp))
    elif args.profile_case == "eq_short":
        import cases
        rng = np.random.default_rng(13)
        for npts in (512, 3000):
            r = np.exp(rng.uniform(np.log(1e4), np.log(5e5), 500))
            u = cases.ricker_records(rng, r, npts, 20.0)
            f = 20.0 * np.arange(200) / npts
            c = np.linspace(2000.0, 5000.0, 400)
            for _ in range(n):
                _quiet(ccfj.fj_earthquake, u, r, c, f)
    else:  # cc_direct
        nsta, npts, fftlen = 50, 86400, 3001
        data = np.random.default_rng(17).standard_normal(nsta * npts, dtype=np.float32)
        se = np.tile([0, npts], nsta).astype(np.int32)
        pairs = ccfj.GetStationPairs(nsta)
        for _ in range(n):
            ccfj.CC(npts, nsta, 500, fftlen, pairs, se, data.copy(), overlaprate=0.5)
    torch.cuda.synchronize()
    print("profile case %s done: %d calls" % (args.profile_case, n))
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
    a = _fj_args(NPAIRS, nf, NC, 1, _lib.MODE_J, d_u.data_ptr(), 2 * NF, 2, d_perm.data_ptr(),
                 d_r, d_f, d_c, d_out)
    if args.profile_case == "hilbert":
        a.mode, a.hilbert = _lib.MODE_J_MINUS_Y, 1
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
    # records to dispersion spectrum in one call (the cross-spectra stay on
    # the device): station coordinates in a 300 x 300 km box, bins at
    # fstride 3 of one-hour windows, 1000 velocities over 2000-5000 m/s (the
    # reference's noise example), itype 1, func 0; host arrays in and out
    xy = np.random.default_rng(8).uniform(0.0, 3e5, (nsta, 2))
    pp = pairs.reshape(-1, 2)
    r = np.hypot(*(xy[pp[:, 0]] - xy[pp[:, 1]]).T)
    fbin = np.arange(nf) * fstride * fs / fftlen
    fbin[0] = fbin[1] / 2  # keep k > 0 in the first column
    cv = np.linspace(2000.0, 5000.0, 1000)
    for _ in range(args.warmup):
        ccfj.cc_fj_noise(npts, nsta, nf, fftlen, pairs, se, data, r, cv, fbin, overlaprate=overlap,
                         fstride=fstride)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ccfj.cc_fj_noise(npts, nsta, nf, fftlen, pairs, se, data, r, cv, fbin, overlaprate=overlap,
                         fstride=fstride)
    chain_s = (time.perf_counter() - t0) / args.steps
    print(json.dumps({
        "case": "cc", "unit": "ms per call", "device_ms": dev_s * 1e3, "e2e_ms": e2e_s * 1e3,
        "records_to_spectrum_ms": chain_s * 1e3,
        "records_to_spectrum": "ccfj.cc_fj_noise on host arrays: the CC above, then fj_noise "
                               "itype 1 func 0 on its %d pairs x %d bins x 1000 velocities; records "
                               "in once (%.0f MB), spectrum out once (%.1f MB)" % (
                                   npairs, nf, data.nbytes / 1e6, 4e-6 * nf * 1000),
        "gpu_launches_per_call": int(launches),
        "algorithmic_tflops": tflops, "fp32_peak_tflops": peak.value,
        "frac_fp32": tflops / peak.value,
        "flops": {"fft": fft_flops, "pair_products": pair_flops},
        "config": {"workload": "CC, reference example day", "nsta": nsta, "npts": npts,
                   "fftlen": fftlen, "steplen": int(a.steplen), "windows": windows, "nf": nf,
                   "fstride": fstride, "npairs": npairs, "l2": "inputs larger than L2"},
        "data": "synthetic (seeded standard normal records)"}))
    return 0


def run_profile_mwfj(args):
    """MWFJ on the configuration-4 traces with fewer windows and bins (for
    ncu captures): 8 windows, 256 bins, func from --profile-case."""
    import torch
    from ccfj import _lib, _eq
    lib = _lib.load()
    wl = workload_mwfj(nf=256, nwin=8)
    u, r, f, c = wl["u"], wl["r"], wl["f"], wl["c"]
    ntr, npts = u.shape
    idx = np.argsort(r)
    n1, n2, dl = _eq._win_params(npts, wl["Fs"], wl["winl"], wl["winr"], wl["taper"])
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=u, perm=idx.astype(np.int64), r=r[idx].astype(np.float32), f=f.astype(np.float32),
        c=c.astype(np.float32), n1=n1.astype(np.int32), n2=n2.astype(np.int32),
        dl=dl.astype(np.int32)).items()}
    out = torch.empty((wl["nwin"], len(c), len(f)), device="cuda")
    a = _eq.EqArgs()
    a.struct_size = ctypes.sizeof(a)
    a.ntr, a.npts, a.nf, a.nc, a.nwin = ntr, npts, len(f), len(c), wl["nwin"]
    a.itype, a.precision, a.normalize, a.device_ptrs, a.fstride = 1, 0, 1, 1, 1
    a.func = 1 if args.profile_case == "mwfj_cc" else 0
    a.u, a.u_ld, a.u_rows = d["u"].data_ptr(), npts, ntr
    a.perm, a.r, a.f, a.c = (d[k].data_ptr() for k in ("perm", "r", "f", "c"))
    a.win_n1, a.win_n2, a.win_delta = (d[k].data_ptr() for k in ("n1", "n2", "dl"))
    a.out = out.data_ptr()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(args.warmup + args.steps):
        _lib.check(lib.ccfj_fj_earthquake_v1(ctypes.byref(a), sp))
    torch.cuda.synchronize()
    print("profile case done: %d MWFJ calls (%d windows, %d bins)" % (
        args.warmup + args.steps, wl["nwin"], len(f)))
    return 0


def run_config(args):
    """One configuration alone (device, end to end, FP64; no CPU sample):
    one JSON line."""
    import torch
    from ccfj import _lib
    lib = _lib.load()
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    peak = ctypes.c_double(0)
    _lib.check(lib.ccfj_fp32_peak_probe(sp, ctypes.byref(peak)))
    dev = torch.cuda.current_device()
    if args.config == 1:
        run = measure_small(lib, torch, dev, sp, peak.value, args)
    elif args.config == 3:
        run = measure_eq(lib, torch, dev, sp, peak.value, args)
    elif args.config == 4:
        run = measure_mwfj(lib, torch, dev, sp, peak.value, bf16_peak(), args)
    else:
        run = measure_batch(lib, torch, dev, sp, peak.value, args)
    print(json.dumps(dict(run.res, config_id=args.config)))
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
    ap.add_argument("--headline-only", action="store_true",
                    help="report the headline workload without the `configs` object")
    ap.add_argument("--profile-case", nargs="?", const="noise", default=None,
                    choices=("noise", "hilbert", "mwfj", "mwfj_cc", "batch", "cc", "noise0",
                             "eq_short", "small", "cc_direct"),
                    help="run a reduced case for ncu captures: 'noise' = the device transform "
                         "on the first 512 frequencies of the workload (steps launches, no "
                         "extras); 'mwfj' = the MWFJ configuration with 8 windows and 256 bins; "
                         "'hilbert' = the same with func 1 (device Hilbert transform); 'mwfj_cc' "
                         "= the MWFJ case with func 1 (CUDA-core kernel); 'batch' = the ragged "
                         "batch with 64 subarrays; 'cc' = cross-correlation of the reference "
                         "example's day (one JSON line); noise0, eq_short, small, cc_direct: "
                         "see run_profile_extra")
    ap.add_argument("--config", type=int, default=0, choices=(0, 1, 3, 4, 5),
                    help="measure one other workload alone (one JSON line): 1 small noise array, "
                         "3 earthquake, 4 MWFJ, 5 ragged batch")
    args = ap.parse_args()
    if args.config:
        return run_config(args)
    if args.profile_case in ("mwfj", "mwfj_cc"):
        return run_profile_mwfj(args)
    if args.profile_case == "cc":
        return run_cc_case(args)
    if args.profile_case in ("noise0", "eq_short", "small", "cc_direct"):
        return run_profile_extra(args)
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
