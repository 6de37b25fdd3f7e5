#!/usr/bin/env python3
"""Regenerates the golden fixtures in this directory by running the
REFERENCE's own CPU implementation (src/ccfj.pyx + src/FJcpu.cpp, built by
`make -C oracle` into oracle/_ref/) on small seeded inputs.

The reference ships no tests, fixtures or example data for the F-J path, so
these files are the only record of its outputs; tests/ pins the FP64 oracle
and the CUDA path against them. Run in a container that has the reference
sources and the oracle/_ref build:

    make -C oracle && python tests/golden/make_golden.py
"""
import ctypes
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle", "_ref"))
sys.path.insert(0, os.path.join(REPO, "tests"))

import ccfj_ref  # noqa: E402  (the reference's Cython module)
from cases import (eq_case, mwfj_case, noise_case)  # noqa: E402


class _Quiet:
    """Silences the reference's stdout prints (trap_J writes f[0..9])."""

    def __enter__(self):
        sys.stdout.flush()
        self.fd = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.fd, 1)
        os.close(self.null)
        os.close(self.fd)


def main():
    warnings.simplefilter("ignore")
    nthr = os.cpu_count() or 1
    out = {}
    for name in ("noise_small", "noise_ties", "noise_fstride2", "noise_real64"):
        case = noise_case(name)
        for itype in (0, 1):
            for func in (0, 1):
                with _Quiet():
                    y = ccfj_ref.fj_noise(case["uf"], case["r"], case["c"], case["f"],
                                          fstride=case["fstride"], itype=itype, func=func, num=nthr)
                out["%s_i%d_f%d" % (name, itype, func)] = np.asarray(y)
    case = eq_case("eq_small")
    for itype in (0, 1):
        for func in (0, 1):
            with _Quiet():
                y = ccfj_ref.fj_earthquake(case["u"], case["r"], case["c"], case["f"],
                                           itype=itype, func=func, num=nthr)
            out["eq_small_i%d_f%d" % (itype, func)] = np.asarray(y)
    case = mwfj_case("mwfj_small")
    for func in (0, 1):
        with _Quiet():
            y = ccfj_ref.MWFJ(case["u"], case["r"], case["c"], case["f"], case["Fs"], case["nwin"],
                              case["winl"], case["winr"], taper=case["taper"], func=func, num=nthr)
        out["mwfj_small_i1_f%d" % func] = np.asarray(y)
    # raw C-ABI outputs of FJ / FH (no sorting, no normalisation)
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libfjcpu.so"))
    fp = ctypes.POINTER(ctypes.c_float)
    for fn in (lib.FJ, lib.FH):
        fn.argtypes = [fp] * 5 + [ctypes.c_int] * 5
        fn.restype = ctypes.c_int
    case = noise_case("raw_small")
    U = np.ascontiguousarray(np.real(case["uf"]), dtype=np.float32)
    r32, f32, c32 = (np.ascontiguousarray(case[k], dtype=np.float32) for k in ("r", "f", "c"))
    nr, nf, nc = len(r32), len(f32), len(c32)
    P = lambda a: a.ctypes.data_as(fp)  # noqa: E731
    for fname, fn in (("FJ", lib.FJ), ("FH", lib.FH)):
        for itype in (0, 1):
            y = np.zeros(nc * nf, dtype=np.float32)
            with _Quiet():
                fn(P(U), P(r32), P(f32), P(y), P(c32), nc, nr, nf, itype, nthr)
            out["raw_%s_i%d" % (fname, itype)] = y.reshape(nc, nf)
    path = os.path.join(HERE, "reference_outputs.npz")
    np.savez_compressed(path, **out)
    print("wrote %s (%d arrays)" % (path, len(out)))


if __name__ == "__main__":
    main()
