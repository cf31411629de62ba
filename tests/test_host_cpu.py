"""CPU-only checks of the shipped library: it loads, exports every function
include/*.h declares, and without a GPU its entry points fail loudly."""
import os
import re

import pytest

from conftest import ROOT
from hartreefock_b200 import engine as E
from hartreefock_b200 import scf


def declared_functions():
    names = set()
    for h in ("hfgpu.h", "hfgpu_driver.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(hf[gd]_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = E.library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(E.EXPORTED + scf.DRIVER_SYMBOLS) <= set(names)


def test_no_device_is_reported_not_hidden():
    # this container has no GPU: creating a context must fail loudly
    if E.library().hfg_device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(E.HfgError):
        E.Engine([1, 1], [[0, 0, 0], [0, 0, 1.4]], "sto-3g")


def test_one_electron_without_device_fails_loudly():
    if E.library().hfg_device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(E.HfgError):
        E.one_electron([1, 1], [[0, 0, 0], [0, 0, 1.4]], "sto-3g")
