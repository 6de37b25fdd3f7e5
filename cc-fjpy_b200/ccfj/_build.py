"""Builds the ccfj_b200 CUDA library in-tree for sm_100a.

    python -m ccfj._build          (from cc-fjpy_b200/)  or  ccfj._build.build()

Every .cu directly under cc-fjpy_b200/csrc is compiled with nvcc for
compute_100a/sm_100a and linked into ccfj/_lib/libccfj_b200.so, which the
Python package loads with ctypes. The unit tests' special-function probe
(csrc/testprobe/) is linked separately into ccfj/_lib/libccfj_b200_probe.so;
the product library does not contain it. Objects go to cc-fjpy_b200/_build/.

Rebuilds are decided by content, not by file times: every object records a
SHA-256 of its source, all headers, the compiler flags and the nvcc version,
and the library records the digest of its objects beside itself
(libccfj_b200.so.sha256). A library whose recorded digest differs from the
current sources is rebuilt before it is loaded, so a copied tree never runs a
binary built from other sources.
"""
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)                      # cc-fjpy_b200/
CSRC = os.path.join(ROOT, "csrc")
PROBE_SRC = os.path.join(CSRC, "testprobe")
OBJ = os.path.join(ROOT, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libccfj_b200.so")
PROBE_LIB = os.path.join(LIBDIR, "libccfj_b200_probe.so")
INCLUDE = os.path.join(os.path.dirname(ROOT), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC,
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build ccfj_b200")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def probe_sources():
    return sorted(os.path.join(PROBE_SRC, f) for f in os.listdir(PROBE_SRC) if f.endswith(".cu"))


def _headers():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return sorted(hdrs)


_NVCC_VERSION = None


def _nvcc_version():
    global _NVCC_VERSION
    if _NVCC_VERSION is None:
        try:
            _NVCC_VERSION = subprocess.run([nvcc(), "--version"], capture_output=True,
                                           text=True).stdout
        except (OSError, RuntimeError):
            _NVCC_VERSION = "unknown"
    return _NVCC_VERSION


def _digest(paths, extra=""):
    h = hashlib.sha256()
    for p in paths:
        h.update(os.path.relpath(p, ROOT).encode())
        with open(p, "rb") as fh:
            h.update(fh.read())
    h.update(extra.encode())
    return h.hexdigest()


def _object_digest(src):
    return _digest([src] + _headers(), " ".join(NVCC_FLAGS) + _nvcc_version())


def _read(path):
    try:
        with open(path) as fh:
            return fh.read().strip()
    except OSError:
        return None


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    dg = _object_digest(src)
    if os.path.exists(obj) and _read(obj + ".sha256") == dg and not verbose:
        return obj, dg, ""
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), p.stderr))
    with open(obj + ".sha256", "w") as fh:
        fh.write(dg)
    return obj, dg, p.stderr


def expected_digest(srcs):
    """Digest a library built from `srcs` records (no compilation)."""
    return hashlib.sha256("".join(_object_digest(s) for s in srcs).encode()).hexdigest()


def up_to_date(lib=LIB, srcs=None):
    srcs = sources() if srcs is None else srcs
    return os.path.exists(lib) and _read(lib + ".sha256") == expected_digest(srcs)


def _link(lib, srcs, verbose):
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if verbose:
        for _, _, log in results:
            if log:
                sys.stderr.write(log)
    dg = hashlib.sha256("".join(d for _, d, _ in results).encode()).hexdigest()
    if os.path.exists(lib) and _read(lib + ".sha256") == dg:
        return lib
    tmp = lib + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + [o for o, _, _ in results] + ["-lcudart"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), p.stderr))
    os.replace(tmp, lib)
    with open(lib + ".sha256", "w") as fh:
        fh.write(dg)
    return lib


def build(verbose=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            os.remove(os.path.join(OBJ, f))
        for lib in (LIB, PROBE_LIB):
            if os.path.exists(lib + ".sha256"):
                os.remove(lib + ".sha256")
    _link(LIB, sources(), verbose)
    _link(PROBE_LIB, probe_sources(), verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
