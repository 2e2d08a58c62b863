"""GPU chemistry chain against the oracle: RHF, CCSD, RDMs, the full CCSD
gradient (oracle pinned to central finite differences) and the autograd path."""
import os

import numpy as np
import pytest
import torch

from oracle import cc_oracle as C
from oracle import scf_cc_oracle as Q
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _tensor_cores_at_small_sizes(monkeypatch):
    """These systems are small enough that every contraction would take the
    launch-bound FP64 route; keep the split-precision modes on the tensor cores."""
    import ccsd_gpu_b200.contract as Cn
    monkeypatch.setattr(Cn, "SMALL_FLOPS", 0.0)
    monkeypatch.setattr(Cn, "MIXED_MIN_LADDER_FLOPS", 0.0)

H2O = "O 0 0 0; H 0 -0.757 0.587; H 0.05 0.757 0.587"


@pytest.fixture(scope="module")
def h2o_oracle():
    from ccsd_gpu_b200.gto import M
    mol = M(atom=H2O, basis="cc-pvdz")
    mf, eris, etot, t1, t2 = Q.ccsd_total(mol)
    l1, l2 = Q.lambda_solve(t1, t2, eris)
    g = Q.grad_elec(mf, t1, t2, l1, l2) + mol.grad_nuc()
    return dict(mol=mol, mf=mf, etot=etot, t1=t1, t2=t2, l1=l1, l2=l2, grad=g)


def test_rhf_energy_matches_oracle(h2o_oracle):
    from ccsd_gpu_b200.scf import RHF
    mf = RHF(h2o_oracle["mol"]).run()
    assert mf.converged
    assert abs(mf.e_tot - h2o_oracle["mf"].e_tot) < 1e-9


@pytest.mark.parametrize("mode,tol", [("fp64", 1e-9), ("tf32x3", 1e-7)])
def test_ccsd_energy_matches_oracle(h2o_oracle, mode, tol):
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.scf import RHF
    cc = CCSD(RHF(h2o_oracle["mol"]).run(), precision=mode)
    cc.kernel()
    assert cc.converged
    assert abs(cc.e_tot - h2o_oracle["etot"]) < tol


@pytest.mark.parametrize("fixture", ["cc_small.npz", "cc_blocked.npz"])
@pytest.mark.parametrize("mode,tol", [("fp64", 1e-12), ("tf32x3", 5e-6)])
def test_rdm_intermediates_match_reference_golden(mode, tol, fixture):
    from types import SimpleNamespace
    from ccsd_gpu_b200 import gpu_ccsd_grad as G
    d = dict(np.load(os.path.join(GOLDEN, fixture)))
    cc = SimpleNamespace(precision=mode)
    args = (d["t1"], d["t2"], d["l1"], d["l2"])
    rel = lambda a, b: float(np.abs(a.cpu().numpy() - b).max() / np.abs(b).max())   # noqa: E731
    for k, a in zip(("doo", "dov", "dvo", "dvv"), G._gamma1_intermediates_gpu(cc, *args)):
        assert rel(a, d[k]) < tol, k
    d2 = G._gamma2_intermediates_gpu(cc, *args)
    for k, a in zip(("dovov", "dvvvv", "doooo", "doovv", "dovvo", "dvvov", "dovvv", "dooov"), d2):
        if a is not None:
            assert rel(a, d[k]) < tol, k
    assert rel(G._rdm2_mo2ao_gpu(cc, d2, d["mo_coeff"]), d["dm2_tril"]) < tol


@pytest.mark.parametrize("mode,polish,tol", [("fp64", True, 1e-7), ("tf32x3", True, 1e-6),
                                              ("tf32x3", False, 1e-6), ("bf16x3", True, 1e-6)])
def test_ccsd_gradient_matches_oracle(h2o_oracle, mode, polish, tol):
    """Mixed precision with and without the FP64 polish of the Lambda solve,
    against the FP64 oracle: the north-star bar is max|dg| <= 1e-6 Eh/bohr."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.scf import RHF
    cc = CCSD(RHF(h2o_oracle["mol"]).run(), precision=mode)
    cc.kernel()
    cc.conv_tol_normt = 1e-9
    cc.lambda_polish = polish
    cc.solve_lambda()
    if polish or mode == "fp64":
        assert cc.converged_lambda
    else:
        # stopped at the split-precision floor: not converged to 1e-9, and says so
        assert not cc.converged_lambda and cc.lambda_normt < 1e-6
    g = cc.nuc_grad_method().kernel()
    assert np.abs(g - h2o_oracle["grad"]).max() < tol
    assert np.abs(g.sum(0)).max() < 1e-8


def test_compute_ml_ccsd_forces_gpu_with_oracle_amplitudes(h2o_oracle):
    from ccsd_gpu_b200.gpu_ccsd_grad import compute_ml_ccsd_forces_gpu
    from ccsd_gpu_b200.scf import RHF
    o = h2o_oracle
    mf = RHF(o["mol"]).run()
    # the amplitudes belong to the oracle's orbitals (MO signs are arbitrary per SCF run)
    mf.mo_coeff, mf.mo_energy = o["mf"].mo_coeff, o["mf"].mo_energy
    g = compute_ml_ccsd_forces_gpu(mf, o["t1"], o["t2"], o["l1"], o["l2"], precision="fp64")
    assert np.abs(g - o["grad"]).max() < 1e-7


def test_autograd_energy_backward_and_finite_difference():
    from ccsd_gpu_b200.gpu_ccsd_grad import CCSDEnergy
    from ccsd_gpu_b200.gto import M
    mol = M(atom=H2O, basis="sto-3g")
    x = torch.tensor(mol.atom_coords(), dtype=torch.float64, device="cuda", requires_grad=True)
    e = CCSDEnergy.apply(x, mol, "fp64")
    e.backward()
    h = 1e-3
    for a, c in [(0, 2), (2, 0)]:
        xs = []
        for s in (1, -1):
            y = x.detach().clone()
            y[a, c] += s * h
            xs.append(float(CCSDEnergy.apply(y, mol, "fp64")))
        assert abs((xs[0] - xs[1]) / (2 * h) - float(x.grad[a, c])) < 5e-7


@pytest.mark.parametrize("mode", ["fp64", "tf32x3"])
def test_cuda_graph_replay_matches_eager(mode):
    """The T and Lambda updates replayed as CUDA graphs give the eager results."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    mf = RHF(M(atom=H2O, basis="cc-pvdz")).run()
    out = {}
    for graphs in (False, True):
        cc = CCSD(mf, precision=mode)
        cc.use_graphs = graphs
        cc.kernel()
        cc.conv_tol_normt = 1e-9
        cc.solve_lambda()
        out[graphs] = (cc.e_tot, cc.nuc_grad_method().kernel())
    assert abs(out[True][0] - out[False][0]) < 1e-10
    assert np.abs(out[True][1] - out[False][1]).max() < 1e-9


def test_nh3_gradient_matches_oracle_fp64_and_mixed():
    """A second molecule (N with a d shell, three H) through the whole chain."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    mol = M(atom="N 0 0 0.12; H 0 0.94 -0.28; H 0.81 -0.47 -0.28; H -0.80 -0.46 -0.30", basis="cc-pvdz")
    _, g_ref = Q.ccsd_gradient(mol)
    for mode, tol in (("fp64", 1e-7), ("tf32x3", 1e-6)):
        cc = CCSD(RHF(mol).run(), precision=mode)
        cc.kernel()
        cc.conv_tol_normt = 1e-9
        g = cc.nuc_grad_method().kernel()
        assert np.abs(g - g_ref).max() < tol, (mode, np.abs(g - g_ref).max())


def test_frozen_core_gradient_matches_finite_differences():
    """Frozen O 1s: analytic gradient (active-space RDMs, frozen-active block
    of the relaxed density) against central differences of the frozen-core
    energy, step 1e-3 bohr on all nine coordinates; mixed vs FP64 <= 1e-6."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    mol = M(atom=H2O, basis="cc-pvdz")

    def energy(m):
        cc = CCSD(RHF(m).run(), precision="fp64", frozen=1)
        cc.conv_tol = 1e-11
        cc.conv_tol_normt = 1e-9
        cc.kernel()
        return cc.e_tot

    grads = {}
    for mode in ("fp64", "tf32x3"):
        cc = CCSD(RHF(mol).run(), precision=mode, frozen=1)
        cc.kernel()
        cc.conv_tol_normt = 1e-9
        assert cc.t1.shape == (4, 19)
        grads[mode] = cc.nuc_grad_method().kernel()
    x0 = mol.atom_coords()
    h = 1e-3
    fd = np.zeros_like(x0)
    for a in range(mol.natm):
        for c in range(3):
            ep = []
            for sgn in (1, -1):
                x = x0.copy()
                x[a, c] += sgn * h
                ep.append(energy(mol.copy().set_geom_(x)))
            fd[a, c] = (ep[0] - ep[1]) / (2 * h)
    assert np.abs(grads["fp64"] - fd).max() < 1e-6, np.abs(grads["fp64"] - fd).max()
    assert np.abs(grads["tf32x3"] - grads["fp64"]).max() < 1e-6
    assert np.abs(grads["fp64"].sum(0)).max() < 1e-8


def test_cached_fp64_solve_graphs_match_eager_across_geometries():
    """FP64 T/Lambda bodies replayed from the cross-solve graph cache: a second
    geometry (new integrals copied into the captured tensors) gives the eager
    energy and gradient."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.graphs import clear_solve_graphs
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    clear_solve_graphs()
    geoms = [H2O, "O 0 0 0.02; H 0 -0.74 0.60; H 0.03 0.77 0.57"]
    for atom in geoms:
        mf = RHF(M(atom=atom, basis="cc-pvdz")).run()
        out = {}
        for cached in (True, False):
            cc = CCSD(mf, precision="fp64")
            cc.use_graph_cache = cached
            cc.kernel()
            cc.conv_tol_normt = 1e-9
            cc.solve_lambda()
            out[cached] = (cc.e_tot, cc.nuc_grad_method().kernel())
        assert abs(out[True][0] - out[False][0]) < 1e-10
        assert np.abs(out[True][1] - out[False][1]).max() < 1e-9


def test_cached_split_precision_solve_graphs_match_eager_across_geometries():
    """The same for tf32x3 bodies: packs of the integrals are graph nodes, so a
    second geometry replays with its own integrals."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.graphs import clear_solve_graphs
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    clear_solve_graphs()
    for atom in (H2O, "O 0 0 0.02; H 0 -0.74 0.60; H 0.03 0.77 0.57"):
        mf = RHF(M(atom=atom, basis="cc-pvdz")).run()
        out = {}
        for cached in (True, False):
            cc = CCSD(mf, precision="tf32x3")
            cc.use_graph_cache = cached
            cc.t_polish = cc.lambda_polish = False
            cc.kernel()
            cc.conv_tol_normt = 1e-9
            cc.solve_lambda()
            out[cached] = (cc.e_tot, cc.nuc_grad_method().kernel())
        assert abs(out[True][0] - out[False][0]) < 1e-9
        assert np.abs(out[True][1] - out[False][1]).max() < 1e-8


def test_device_amplitude_hand_off_matches_host_arrays(h2o_oracle):
    """The solves keep device copies of t1/t2/l1/l2 next to their (read-only)
    host arrays; the gradient from that hand-off equals the one from fresh
    host copies, which take the upload path."""
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.scf import RHF
    cc = CCSD(RHF(h2o_oracle["mol"]).run(), precision="fp64")
    cc.kernel()
    cc.conv_tol_normt = 1e-9
    cc.solve_lambda()
    for a in (cc.t1, cc.t2, cc.l1, cc.l2):
        assert not a.flags.writeable
    g_dev = cc.nuc_grad_method().kernel()
    g_host = cc.nuc_grad_method().kernel(*(np.array(a) for a in (cc.t1, cc.t2, cc.l1, cc.l2)))
    assert np.abs(g_dev - g_host).max() < 1e-12
    assert np.abs(g_dev - h2o_oracle["grad"]).max() < 1e-7
