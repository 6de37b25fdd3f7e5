"""Cross-spectra files: the `.npz` hand-off between CC and fj_noise.

The reference's workflow stores the stacked cross-spectra with
np.savez(name, ncfs=..., r=..., f=...) and reads them back with np.load
before fj_noise (examples/example_noise.py:6-11; the notebook
examples/example_CC.ipynb writes them). load_ncfs reads such a file with
the spectra landing directly in page-locked (pinned) host memory, from
which the transform's upload is a DMA without a staging copy.
"""
import ctypes
import weakref
import zipfile

import numpy as np

from . import _lib

_lib.SIGNATURES["ccfj_host_alloc"] = (ctypes.c_int, [ctypes.c_size_t,
                                                      ctypes.POINTER(ctypes.c_void_p)])
_lib.SIGNATURES["ccfj_host_free"] = (ctypes.c_int, [ctypes.c_void_p])


def pinned_empty(shape, dtype):
    """An uninitialised numpy array in page-locked host memory (freed when
    the array and every view of it are gone)."""
    lib = _lib.load()
    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
    ptr = ctypes.c_void_p()
    _lib.check(lib.ccfj_host_alloc(max(nbytes, 1), ctypes.byref(ptr)))
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(ptr.value)
    weakref.finalize(buf, lib.ccfj_host_free, ptr)
    return np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape, dtype=np.int64))).reshape(
        shape)


def _read_member_into(zf, name):
    """Reads one .npy member of an open zip into pinned memory: header
    parsed, data read straight into the buffer."""
    with zf.open(name) as fh:
        version = np.lib.format.read_magic(fh)
        if version == (1, 0):
            shape, fortran, dtype = np.lib.format.read_array_header_1_0(fh)
        else:
            shape, fortran, dtype = np.lib.format.read_array_header_2_0(fh)
        if dtype.hasobject:
            raise ValueError("%s holds Python objects" % name)
        arr = pinned_empty(shape if not fortran else shape[::-1], dtype)
        view = memoryview(arr.reshape(-1).view(np.uint8))
        got = 0
        while got < len(view):
            n = fh.readinto(view[got:])
            if not n:
                raise ValueError("%s: file ends after %d of %d bytes" % (name, got, len(view)))
            got += n
    return arr.T if fortran else arr


def load_ncfs(path, keys=("ncfs", "r", "f")):
    """Loads the cross-spectra file written by np.savez(path, ncfs=..., r=...,
    f=...): a dict of numpy arrays, each in pinned host memory, read
    member by member without an intermediate copy (compressed members are
    decompressed in stream). Keys other than `keys` are not read."""
    out = {}
    with zipfile.ZipFile(path) as zf:
        names = {n[:-4]: n for n in zf.namelist() if n.endswith(".npy")}
        for k in keys:
            if k not in names:
                raise KeyError("%s is not a file in the archive %s" % (k, path))
            out[k] = _read_member_into(zf, names[k])
    return out
