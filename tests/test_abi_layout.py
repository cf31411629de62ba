"""The ctypes mirrors of the C ABI structs (engine.py, scf.py) have the same
size and field offsets as the C declarations in include/*.h, checked by
compiling a probe against the headers with the system C compiler."""
import ctypes
import os
import subprocess
import tempfile

import pytest

from conftest import ROOT
from hartreefock_b200 import engine as E
from hartreefock_b200 import scf
from hartreefock_b200 import serve

STRUCTS = [("hfg_shells", E.hfg_shells), ("hfg_opts", E.hfg_opts), ("hfg_stats", E.hfg_stats),
           ("hfg_class_time", E.hfg_class_time), ("hfd_scf_opts", scf.hfd_scf_opts),
           ("hfd_scf_result", scf.hfd_scf_result), ("hfg_job_spec", serve.hfg_job_spec),
           ("hfg_job_info", serve.hfg_job_info)]


def _c_layout():
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "hfgpu_driver.h"', "int main(void) {"]
    for cname, cls in STRUCTS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "probe.c"), os.path.join(d, "probe")
        with open(src, "w") as fh:
            fh.write("\n".join(lines))
        r = subprocess.run(["gcc", "-std=c99", "-I" + os.path.join(ROOT, "include"), src, "-o", exe],
                           capture_output=True, text=True)
        if r.returncode != 0:
            pytest.fail(r.stderr)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    layout = {}
    for line in out.splitlines():
        a, b, v = line.split()
        layout[(a, b)] = int(v)
    return layout


def test_ctypes_structs_match_headers():
    layout = _c_layout()
    for cname, cls in STRUCTS:
        assert ctypes.sizeof(cls) == layout[(cname, "size")], cname
        for f, _ in cls._fields_:
            assert getattr(cls, f).offset == layout[(cname, f)], (cname, f)
