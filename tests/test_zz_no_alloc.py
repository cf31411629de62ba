"""The allocation-free entry point hfg_fock_rhf_noalloc, called through the C
ABI, against the allocating hfg_fock_rhf_device on the same density.

It serves callers that cannot allocate device memory on their hot path;
its J/K scratch is a fixed 16 MiB device array shared by all calls.  Two
calls in a row check that the second one starts from cleared accumulators.
This file is collected last so that a failure here stops a run only after
every other test has run."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,convention", [("h2o2_631gs", "reference"), ("o2_631gs", "reference"),
                                             ("o2_631gs", "exact")])
def test_noalloc_fock_matches_allocating_entry_point(name, convention):
    """Both ERI conventions, on molecules whose d shells reach every class up
    to (dd|dd) (O2: two-centre d pairs)."""
    import torch
    from hartreefock_b200 import engine as E
    g = load_golden(name)
    conv = E.ERI_REFERENCE if convention == "reference" else E.ERI_EXACT
    eng = E.Engine(list(g["Z"]), g["xyz"], str(g["basis"]), schwarz_threshold=1e-12, eri_convention=conv)
    n = eng.nbf
    rng = np.random.default_rng(7)
    A = rng.normal(size=(n, n)) * 0.1
    P = torch.from_numpy(A + A.T).cuda()
    G_ref = torch.empty_like(P)
    stream = E._torch_stream()  # torch's stream: ordered with the fills and copies below
    eng.fock_rhf_device(P.data_ptr(), G_ref.data_ptr(), stream)
    torch.cuda.synchronize()
    want = G_ref.cpu().numpy()
    scale = max(1.0, float(np.abs(want).max()))
    for _ in range(2):
        G = torch.full_like(P, float("nan"))
        eng.fock_rhf_noalloc(P.data_ptr(), G.data_ptr(), stream)
        torch.cuda.synchronize()
        got = G.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.abs(got - want).max() < 1e-10 * scale
    eng.close()


def test_noalloc_rejects_contexts_above_its_scratch():
    from hartreefock_b200 import engine as E
    from hartreefock_b200 import molecules
    Z, xyz = molecules.water_cluster(54, seed=0)  # 1026 basis functions in 6-31G*
    eng = E.Engine(Z, xyz, "6-31g*", schwarz_threshold=1e-10)
    assert eng.nbf > 1024
    with pytest.raises(E.HfgError, match="exceed"):
        eng.fock_rhf_noalloc(0x1000, 0x1000)
    eng.close()


def test_noalloc_rejects_precision_form_contexts():
    from hartreefock_b200 import engine as E
    g = load_golden("h2o_631gs")
    eng = E.Engine(list(g["Z"]), g["xyz"], str(g["basis"]), schwarz_threshold=1e-12)
    eng.set_mixed_cutoff(1e-4)
    with pytest.raises(E.HfgError, match="precision-form"):
        eng.fock_rhf_noalloc(0x1000, 0x1000)
    eng.close()
