"""The CCSD gradient assembly against the reference's own grad_elec_gpu.

tests/golden/grad_h2o_ccpvdz.npz holds the electronic gradient that the
reference's grad_elec_gpu (ccsd_gpu/gpu_ccsd_grad.py:344-586) computes on the
CPU for H2O/cc-pVDZ, all-electron and with the O 1s orbital frozen, together
with the orbitals and amplitudes it was given (tests/golden/make_grad_golden.py).
The oracle's restatement and the GPU path are checked on the same inputs."""
import os

import numpy as np
import pytest

from tests.conftest import GOLDEN


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLDEN, "grad_h2o_ccpvdz.npz")))


def _amps(d, tag):
    return tuple(d[tag + "_" + k] for k in ("t1", "t2", "l1", "l2"))


@pytest.mark.parametrize("tag", ["fc0", "fc1"])
def test_oracle_assembly_matches_reference(gold, tag):
    from ccsd_gpu_b200.gto import M
    from oracle import scf_cc_oracle as Q
    mol = M(atom=str(gold["atom"]), basis=str(gold["basis"]))
    mf = Q.rhf(mol)
    assert abs(mf.e_tot - float(gold["e_hf"])) < 1e-9
    mf.mo_coeff, mf.mo_energy = gold["mo_coeff"], gold["mo_energy"]
    g = Q.grad_elec(mf, *_amps(gold, tag))
    assert np.abs(g - gold[tag + "_de"]).max() < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["fc0", "fc1"])
@pytest.mark.parametrize("mode,tol", [("fp64", 1e-9), ("tf32x3", 1e-6)])
def test_gpu_gradient_matches_reference(gold, tag, mode, tol, monkeypatch):
    """compute_ml_ccsd_forces_gpu (the reference's public entry point) on the
    reference's inputs; tf32x3 keeps its split-precision RDM contractions on
    the tensor cores at this size."""
    import ccsd_gpu_b200.contract as Cn
    from ccsd_gpu_b200.gpu_ccsd_grad import compute_ml_ccsd_forces_gpu
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    monkeypatch.setattr(Cn, "SMALL_FLOPS", 0.0)
    mol = M(atom=str(gold["atom"]), basis=str(gold["basis"]))
    mf = RHF(mol).run()
    assert abs(mf.e_tot - float(gold["e_hf"])) < 1e-9
    mf.mo_coeff, mf.mo_energy = gold["mo_coeff"], gold["mo_energy"]
    g = compute_ml_ccsd_forces_gpu(mf, *_amps(gold, tag), precision=mode)
    ref = gold[tag + "_de"] + gold["grad_nuc"]
    assert np.abs(g - ref).max() < tol
