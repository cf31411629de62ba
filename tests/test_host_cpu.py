"""CPU-only checks of the shipped library: it loads, exports every function
include/*.h declares, and without a GPU its entry points fail loudly."""
import os
import re

import pytest

from conftest import ROOT
from hartreefock_b200 import engine as E
from hartreefock_b200 import scf
from hartreefock_b200 import serve


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
    assert set(E.EXPORTED + scf.DRIVER_SYMBOLS + serve.POOL_SYMBOLS) <= set(names)


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


XYZ_CASES = {
    "water": "3\nwater, coordinates as written\nO 0.0 0.0 0.24026010\nH 0.0 1.43233673 -0.96104039\n"
             "H 0.0 -1.43233673 -0.96104039\n",
    "methane_extra_columns": "5\n\nC 0 0 0 extra\nH 1.18 1.18 1.18\nH -1.18 -1.18 1.18\nH -1.18 1.18 -1.18\n"
                             "H 1.18 -1.18 -1.18\n",
    "short_file": "3\ncomment\nO 0 0 0\nH 0 0 1.8\n",
    "unknown_symbol": "2\n\nXx 0 0 0\nH 0 0 1.8\n",
    "lowercase_symbol": "2\n\no 0 0 0\nh 0 0 1.8\n",
    "not_in_basis": "1\n\nNa 0 0 0\n",
    "bad_count": "two\n\nH 0 0 0\nH 0 0 1.4\n",
}


@pytest.mark.parametrize("case", sorted(XYZ_CASES))
def test_load_xyz_matches_reference(case, tmp_path):
    """Systems::Molecule::LoadXYZ against the reference's own Molecule::LoadXYZ
    (Molecule.cpp:143-199, compiled headless in oracle/_ref/ref_driver) on the
    same file and basis: same atoms, coordinates and function count, and the
    same refusals."""
    import json
    import subprocess
    import oracle as O
    from hartreefock_b200.basis_io import basis_path
    if not os.path.exists(O.DRIVER_PATH):
        pytest.skip("oracle/_ref/ref_driver not built")
    path = tmp_path / f"{case}.xyz"
    path.write_text(XYZ_CASES[case])
    ref = subprocess.run([O.DRIVER_PATH], input=f"basis {basis_path('6-31g*')}\nxyz {path}\nmode xyz\n",
                         capture_output=True, text=True, timeout=60)
    assert ref.returncode == 0, ref.stderr
    want = json.loads(ref.stdout.strip().splitlines()[-1])
    got = scf.load_xyz(str(path), "6-31g*")
    if not want["ok"]:
        assert got is None
        return
    Z, xyz, nbf = got
    assert Z == [a[0] for a in want["atoms"]]
    assert xyz.tolist() == [a[1:] for a in want["atoms"]]
    assert nbf == want["nbf"]
