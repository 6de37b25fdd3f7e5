"""The ctypes mirrors of the C-ABI argument structs match include/ccfj_b200.h
field by field: a small C program compiled with gcc prints sizeof and the
offset of every field, and the ctypes layouts must agree. The library's own
struct_size check catches a size mismatch at run time; this also catches
fields that are reordered or retyped at equal size."""
import os
import shutil
import subprocess
import tempfile

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _structs():
    from ccfj import _batch, _cc, _eq, _lib
    return [("ccfj_fj_args", _lib.FjArgs), ("ccfj_eq_args", _eq.EqArgs),
            ("ccfj_batch_args", _batch.BatchArgs), ("ccfj_cc_args", _cc.CcArgs),
            ("ccfj_cc_data", _cc.CcData)]


def test_ctypes_layouts_match_header():
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include "ccfj_b200.h"', "#include <stddef.h>", "#include <stdio.h>",
             "int main(void) {"]
    expect = []
    for cname, cls in _structs():
        lines.append('  printf("%%zu\\n", sizeof(%s));' % cname)
        expect.append(("sizeof " + cname, ctypes_size(cls)))
        for fname, _ in cls._fields_:
            lines.append('  printf("%%zu\\n", offsetof(%s, %s));' % (cname, fname))
            expect.append(("%s.%s" % (cname, fname), getattr(cls, fname).offset))
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        subprocess.run([cc, "-std=c99", "-I", os.path.join(REPO, "include"), src, "-o", exe],
                       check=True)
        got = [int(x) for x in subprocess.run([exe], check=True, capture_output=True,
                                              text=True).stdout.split()]
    assert len(got) == len(expect)
    bad = [(name, want, c) for (name, want), c in zip(expect, got) if want != c]
    assert not bad, bad


def ctypes_size(cls):
    import ctypes
    return ctypes.sizeof(cls)
