"""Parity at (reduced) benchmark-configuration sizes.

* Ethanol/cc-pVDZ (the autograd configuration: 9 atoms, nao 72, nocc 13):
  CCSDEnergy backward against central finite differences (1e-3 bohr) of the
  FP64 energy, on a seeded subset of 6 of the 27 coordinates, in FP64 and in
  the split-precision mode.
* The Lambda/RDM configuration's synthetic state at reduced size (nocc 8,
  nvir 72 instead of 24, 216): intermediates, Lambda updates and the density
  intermediates against the numpy oracle (which the reference's own code
  pins, tests/test_cc_oracle.py).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ethanol():
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.gto import M
    sym, xyz = workloads.ethanol_atoms(seed=0)
    return M(atom=workloads.atom_string(sym, xyz), basis="cc-pvdz")


def _energy(mol, xyz):
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.scf import RHF
    cc = CCSD(RHF(mol.copy().set_geom_(xyz)).run(), precision="fp64")
    cc.conv_tol, cc.conv_tol_normt = 1e-11, 1e-9
    cc.kernel()
    return cc.e_tot


@pytest.fixture(scope="module")
def ethanol_fd(ethanol):
    h = 1e-3
    x0 = ethanol.atom_coords()
    coords = np.random.default_rng(0).choice(x0.size, 6, replace=False)
    fd = {}
    for c in coords:
        a, x = divmod(int(c), 3)
        e = []
        for s in (1, -1):
            xs = x0.copy()
            xs[a, x] += s * h
            e.append(_energy(ethanol, xs))
        fd[(a, x)] = (e[0] - e[1]) / (2 * h)
    return fd


@pytest.mark.parametrize("mode,tol", [("fp64", 1e-6), ("tf32x3", 1.5e-6)])
def test_ethanol_autograd_backward_matches_finite_differences(ethanol, ethanol_fd, mode, tol):
    from ccsd_gpu_b200.gpu_ccsd_grad import CCSDEnergy
    x = torch.tensor(ethanol.atom_coords(), dtype=torch.float64, device="cuda", requires_grad=True)
    e = CCSDEnergy.apply(x, ethanol, mode)
    e.backward()
    g = x.grad.cpu().numpy()
    assert np.abs(g.sum(0)).max() < 1e-7            # translational invariance
    for (a, c), v in ethanol_fd.items():
        assert abs(g[a, c] - v) < tol, (mode, a, c, g[a, c], v)


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else a
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("mode,tol", [("fp64", 1e-11), ("tf32x3", 2e-5)])
def test_lambda_rdm_reduced_config_matches_oracle(mode, tol, monkeypatch):
    import ccsd_gpu_b200.contract as Cn
    monkeypatch.setattr(Cn, "SMALL_FLOPS", 0.0)       # every contraction of the split mode on the tensor cores
    from types import SimpleNamespace
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.gpu_ccsd_grad import _gamma1_intermediates_gpu, _gamma2_intermediates_gpu
    from ccsd_gpu_b200.gpu_ccsd_lambda import DeviceEris, make_intermediates_gpu, update_lambda_gpu
    from oracle import cc_oracle as C
    eris, t1, t2 = workloads.lambda_bench_state(8, 72, seed=3, device="cuda")
    host = SimpleNamespace(**{k: getattr(eris, k).cpu().numpy() for k in
                              ("fock", "mo_energy", "oooo", "ovoo", "ovvo", "oovv", "ovov", "ovvv", "vvvv")})
    t1h, t2h = t1.cpu().numpy(), t2.cpu().numpy()
    deris = DeviceEris(eris, torch.device("cuda"))
    cc = SimpleNamespace(level_shift=0.0, precision=mode)
    imds = make_intermediates_gpu(cc, t1, t2, deris, mode)
    ref_imds = C.make_intermediates(t1h, t2h, host.fock, host)
    for k in ("w1", "w2", "w3", "w4", "woooo", "wvooo", "wVOov", "wvOOv", "wvvov"):
        assert _rel(getattr(imds, k), getattr(ref_imds, k)) < tol, k
    l1, l2 = t1, t2
    r1, r2 = t1h, t2h
    for _ in range(3):
        l1, l2 = update_lambda_gpu(cc, t1, t2, l1, l2, deris, imds, mode=mode)
        r1, r2 = C.update_lambda(t1h, t2h, r1, r2, host.fock, host.mo_energy, host, ref_imds)
    assert _rel(l1, r1) < tol and _rel(l2, r2) < tol
    for got, ref in zip(_gamma1_intermediates_gpu(cc, t1, t2, l1, l2), C.gamma1(t1h, t2h, r1, r2)):
        assert _rel(got, ref) < tol
    for got, ref in zip(_gamma2_intermediates_gpu(cc, t1, t2, l1, l2), C.gamma2(t1h, t2h, r1, r2)):
        if ref is not None:
            assert _rel(got, ref) < tol
