"""Seeded synthetic inputs shared by the tests, the golden-fixture script and
the benchmark. The reference publishes no data sets for the F-J path (its
example data are not distributed with it), so every case is generated from a
fixed seed with the shapes and value laws of the benchmark configurations:

  noise spectra  uf = J0(2 pi f r / c(f)) (+ overtone) + complex Gaussian noise,
                 c(f) = 2000 + 1500 exp(-f / 0.2) m/s
  earthquake     dispersed Ricker wavelets (fc = 0.1 Hz) group-delayed by
                 r / c(f), plus white noise at SNR 5
"""
import numpy as np
from scipy.special import j0


def c_law(f):
    return 2000.0 + 1500.0 * np.exp(-np.asarray(f) / 0.2)


def noise_spectra(rng, r, f, sigma=0.1, overtone=False, dtype=np.complex64):
    cf = c_law(f)
    U = j0(2 * np.pi * f[None, :] * r[:, None] / cf[None, :])
    if overtone:
        U = U + 0.5 * j0(2 * np.pi * f[None, :] * r[:, None] / (cf[None, :] + 800.0))
    noise = sigma * (rng.standard_normal(U.shape) + 1j * rng.standard_normal(U.shape))
    return (U + noise).astype(dtype)


def noise_case(name):
    """Small fj_noise cases (names used by the golden fixtures)."""
    if name == "noise_small":
        rng = np.random.default_rng(11)
        r = rng.uniform(1e3, 5e4, 60)
        f = np.linspace(0.01, 1.0, 40)
        c = np.linspace(1000, 5000, 50)
        return dict(uf=noise_spectra(rng, r, f), r=r, f=f, c=c, fstride=1)
    if name == "noise_ties":
        rng = np.random.default_rng(12)
        r = rng.uniform(1e3, 3e4, 50)
        r[10:14] = r[3]            # exact ties
        r[20] = r[21] + 0.03       # gaps below the 0.1 m floor
        r[30] = r[31] + 0.07
        f = np.linspace(0.02, 0.8, 24)
        c = np.linspace(1500, 4500, 30)
        return dict(uf=noise_spectra(rng, r, f, sigma=0.2), r=r, f=f, c=c, fstride=1)
    if name == "noise_fstride2":
        rng = np.random.default_rng(13)
        r = rng.uniform(2e3, 4e4, 40)
        f = np.linspace(0.02, 0.9, 20)
        ff = np.linspace(0.02, 0.9 + (f[1] - f[0]) / 2, 40)
        return dict(uf=noise_spectra(rng, r, ff), r=r, f=f, c=np.linspace(1500, 4500, 30),
                    fstride=2)
    if name == "noise_real64":
        rng = np.random.default_rng(14)
        r = rng.uniform(5e2, 2e4, 32)
        f = np.linspace(0.05, 1.0, 16)
        uf = np.real(noise_spectra(rng, r, f, dtype=np.complex128))
        return dict(uf=uf, r=r, f=f, c=np.linspace(1000, 4000, 24), fstride=1)
    if name == "raw_small":
        rng = np.random.default_rng(15)
        r = np.sort(rng.uniform(1e3, 3e4, 30))
        f = np.linspace(0.02, 0.6, 12)
        return dict(uf=noise_spectra(rng, r, f), r=r, f=f, c=np.linspace(1500, 4500, 20),
                    fstride=1)
    raise KeyError(name)


def ricker_records(rng, r, npts, Fs, fc=0.1, snr=5.0, dtype=np.float32):
    """Dispersed Ricker wavelets: every frequency component of a Ricker
    spectrum delayed by r / c(f), plus white noise at the given SNR."""
    nb = npts // 2 + 1
    fb = np.arange(nb) * Fs / npts
    W = (2 / np.sqrt(np.pi)) * fb ** 2 / fc ** 3 * np.exp(-(fb / fc) ** 2)
    cf = c_law(np.maximum(fb, 1e-3))
    phase = np.exp(-2j * np.pi * fb[None, :] * r[:, None] / cf[None, :])
    u = np.fft.irfft(W[None, :] * phase, n=npts, axis=1)
    amp = np.std(u, axis=1, keepdims=True)
    u = u + amp / snr * rng.standard_normal(u.shape)
    return u.astype(dtype)


def eq_case(name):
    if name == "eq_small":
        rng = np.random.default_rng(21)
        npts, Fs = 512, 20.0
        r = np.exp(rng.uniform(np.log(1e4), np.log(2e5), 24))
        nf = 40
        f = Fs * np.arange(nf) / npts
        return dict(u=ricker_records(rng, r, npts, Fs), r=r, f=f, c=np.linspace(2000, 5000, 50),
                    Fs=Fs)
    raise KeyError(name)


def mwfj_case(name):
    if name == "mwfj_small":
        rng = np.random.default_rng(31)
        npts, Fs, ntr, nwin = 256, 10.0, 16, 3
        r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e5), ntr))
        L = rng.integers(40, 200, size=(nwin, ntr))
        start = rng.integers(0, npts - L)
        winl = start / Fs
        winr = (start + L) / Fs
        nf = 24
        f = Fs * np.arange(nf) / npts
        return dict(u=ricker_records(rng, r, npts, Fs), r=r, f=f, c=np.linspace(1500, 5000, 40),
                    Fs=Fs, nwin=nwin, winl=winl, winr=winr, taper=0.9)
    raise KeyError(name)
