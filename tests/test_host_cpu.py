"""CPU-only checks of the shipped library: it loads, exports every function
include/*.h declares, and the host one-electron code (no GPU involved)
reproduces the reference's core Hamiltonian."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden
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


@pytest.mark.parametrize("name", ["h2o_sto3g", "h2o_631gs", "oh_631g", "o2_631gs", "h2o_631ppgss", "h2o2_631gs"])
def test_host_core_hamiltonian_matches_reference(name):
    g = load_golden(name)
    S, h = scf.one_electron(list(g["Z"]), g["xyz"], str(g["basis"]))
    assert np.abs(h - g["h"]).max() < 1e-10
    assert np.abs(np.diag(S) - 1.0).max() < 1e-6  # contracted functions of these sets are near-normalised
