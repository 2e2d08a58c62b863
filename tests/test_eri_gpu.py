"""ERI / ERI-derivative kernels on the GPU against the reference's golden
vectors and the oracle (parity gate, FP64, rtol 1e-10)."""
import os

import numpy as np
import pytest
import torch

from oracle import eri as oracle_eri
from tests.conftest import GOLDEN
from tests.test_oracle import block_close, checksums_close, quartet_nf

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def test_int2e_blocks_match_reference_golden(golden_mols):
    from ccsd_gpu_b200 import compute_int2e_gpu
    for name, (mol, d) in golden_mols.items():
        for b0, b1 in d["blocks"]:
            got = _np(compute_int2e_gpu(mol, int(b0), int(b1)))
            assert block_close(got, d["int2e_%d_%d" % (b0, b1)]), (name, b0, b1)


def test_ip1_blocks_match_reference_golden(golden_mols):
    from ccsd_gpu_b200 import compute_int2e_ip1_gpu
    for name, (mol, d) in golden_mols.items():
        for b0, b1 in d["blocks"]:
            got = _np(compute_int2e_ip1_gpu(mol, int(b0), int(b1)))
            assert got.shape == d["ip1_%d_%d" % (b0, b1)].shape
            assert block_close(got, d["ip1_%d_%d" % (b0, b1)]), (name, b0, b1)


@pytest.mark.parametrize("cart", [True, False])
def test_full_h2o_block_matches_oracle(cart):
    from ccsd_gpu_b200 import compute_int2e_gpu, compute_int2e_ip1_gpu
    from ccsd_gpu_b200.gto import M
    mol = M(atom="O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587", basis="cc-pvdz", cart=cart)
    got0 = _np(compute_int2e_gpu(mol, 0, mol.nbas))
    got1 = _np(compute_int2e_ip1_gpu(mol, 0, mol.nbas))
    assert block_close(got0, oracle_eri.s2kl(mol, 0, mol.nbas, 0))
    assert block_close(got1, oracle_eri.s2kl(mol, 0, mol.nbas, 1))


def _full_tensor(s2kl, n):
    k, l = np.tril_indices(n)
    full = np.zeros(s2kl.shape[:-1] + (n, n))
    full[..., k, l] = s2kl
    full[..., l, k] = s2kl
    return full


def test_eri_permutational_symmetry_and_ip1_translation_invariance():
    """(ij|kl) = (ji|kl) = (kl|ij); sum of derivatives over the four centres = 0."""
    from ccsd_gpu_b200 import compute_int2e_gpu, compute_int2e_ip1_gpu
    from ccsd_gpu_b200.gto import M
    mol = M(atom="C 0 0 0; O 0 0 1.2; H 0.9 0 -0.5; H -0.9 0 -0.5", basis="cc-pvdz", cart=False)
    n = mol.nao_nr()
    g = _full_tensor(_np(compute_int2e_gpu(mol, 0, mol.nbas)), n)
    assert np.abs(g - g.transpose(1, 0, 2, 3)).max() < 1e-11
    assert np.abs(g - g.transpose(2, 3, 0, 1)).max() < 1e-11
    d = _full_tensor(_np(compute_int2e_ip1_gpu(mol, 0, mol.nbas)), n)
    s = d + d.transpose(0, 2, 1, 3, 4) + d.transpose(0, 3, 4, 1, 2) + d.transpose(0, 3, 4, 2, 1)
    assert np.abs(s).max() < 1e-10 * np.abs(d).max()


def test_quartets_up_to_g_match_reference_golden():
    from ccsd_gpu_b200.cuda.quartets import DeviceShells, quartet_checksums
    from ccsd_gpu_b200.workloads import ShellSet
    d = dict(np.load(os.path.join(GOLDEN, "eri_quartets_l4.npz")))
    ds = DeviceShells(ShellSet(d["atm"], d["bas"], d["env"]))
    q = torch.from_numpy(d["quartets"]).cuda()
    nf = quartet_nf(d["bas"], d["quartets"])
    assert checksums_close(_np(quartet_checksums(ds, q, 0)), d["int2e"], nf)
    assert checksums_close(_np(quartet_checksums(ds, q, 1)), d["ip1"], nf)


def test_bench_workload_sample_matches_oracle():
    """4096 synthetic shells (s:p:d = 4:3:2, 1-6 primitives), Schwarz-screened sample."""
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.cuda.quartets import DeviceShells, quartet_checksums, schwarz_bounds
    sh = workloads.eri_bench_shells(4096, seed=0)
    ds = DeviceShells(sh)
    q = workloads.sample_quartets(sh, 3000, seed=3, schwarz_fn=lambda p: schwarz_bounds(ds, p))
    qd = torch.from_numpy(q).cuda()
    nf = quartet_nf(sh._bas, q)
    for deriv in (0, 1):
        got = _np(quartet_checksums(ds, qd, deriv))
        assert checksums_close(got, oracle_eri.quartet_checksums(sh, q, deriv), nf), deriv


def test_water_dimer_blocks_with_screened_primitive_pairs_match_oracle():
    """Intermolecular shell pairs of a water dimer (cc-pVDZ, O 1s exponents up
    to 1.2e4) lose most primitive pairs to the kernels' pair screen; the blocks
    still equal the unscreened oracle to rtol 1e-10."""
    from ccsd_gpu_b200 import compute_int2e_gpu, compute_int2e_ip1_gpu, workloads
    from ccsd_gpu_b200.gto import M
    cl = workloads.water_clusters(64, seed=0)
    s, x = next(c for c in cl if len(c[0]) == 6)
    mol = M(atom=workloads.atom_string(s, x), basis="cc-pvdz")
    for b0, b1 in [(0, 2), (11, 13), (mol.nbas - 3, mol.nbas)]:
        assert block_close(_np(compute_int2e_gpu(mol, b0, b1)), oracle_eri.s2kl(mol, b0, b1, 0)), (b0, b1)
        assert block_close(_np(compute_int2e_ip1_gpu(mol, b0, b1)), oracle_eri.s2kl(mol, b0, b1, 1)), (b0, b1)


def test_invalid_arguments_are_rejected_on_host():
    from ccsd_gpu_b200 import _native
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200 import compute_int2e_gpu
    mol = M(atom="H 0 0 0; H 0 0 0.74", basis="sto-3g")
    with pytest.raises(ValueError):
        compute_int2e_gpu(mol, 1, 1)
    with pytest.raises(_native.NativeError):
        _native.call("ccsd_b200_eri_s2kl_cart", 0, None, None, None, 0, None, 0, 0, 0, 0, None, 0, None, None)
    with pytest.raises(_native.NativeError):
        x = torch.zeros(8, dtype=torch.float64, device="cuda")
        _native.call("ccsd_b200_eri_s2kl_cart", 0, _native.ptr(x), _native.ptr(x), _native.ptr(x), 1,
                     _native.ptr(x), 0, 1, 1, 5, None, 0, _native.ptr(x), None)


@pytest.mark.parametrize("cart", [True, False])
def test_dense_eri_from_unique_quartets_matches_s2kl_and_oracle(cart):
    """full_eri_gpu computes each unique shell quartet once and writes all 8
    index orders: it must equal the s2kl path unpacked, and the oracle."""
    from ccsd_gpu_b200 import compute_int2e_gpu
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import full_eri_gpu
    for atom in ("O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587",
                 "C 0 0 0; O 0 0 1.2; H 0.9 0 -0.5; H -0.9 0 -0.5"):
        mol = M(atom=atom, basis="cc-pvdz", cart=cart)
        g = _np(full_eri_gpu(mol))
        n = g.shape[0]
        ref = _full_tensor(_np(compute_int2e_gpu(mol, 0, mol.nbas)), n)
        assert np.abs(g - ref).max() <= 1e-12 * np.abs(ref).max()
        # equal shells write both (i, j) orders: equal up to the last bits
        assert np.abs(g - g.transpose(1, 0, 2, 3)).max() <= 1e-14 * np.abs(g).max()
        assert np.abs(g - g.transpose(2, 3, 0, 1)).max() <= 1e-14 * np.abs(g).max()
        if atom.startswith("O"):
            k, l = np.tril_indices(n)
            assert block_close(g[:, :, k, l], oracle_eri.s2kl(mol, 0, mol.nbas, 0))


@pytest.mark.parametrize("deriv", [0, 1])
def test_fused_spherical_blocks_equal_the_two_pass_transform(deriv, monkeypatch):
    """ccsd_b200_eri_s2kl_sph (spherical blocks written by the ERI kernels
    themselves) equals the Cartesian kernel followed by the separate sparse
    transform, on blocks with d shells on every centre, heavy (dd|dd)
    quartets included."""
    from ccsd_gpu_b200 import compute_int2e_gpu, compute_int2e_ip1_gpu
    from ccsd_gpu_b200.cuda import _eri
    from ccsd_gpu_b200.gto import M
    mol = M(atom="C 0 0 0; O 0 0 1.2; H 0.9 0 -0.5; H -0.9 0 -0.5", basis="cc-pvdz")
    fn = compute_int2e_ip1_gpu if deriv else compute_int2e_gpu
    for b0, b1 in [(0, 3), (4, 6), (mol.nbas - 4, mol.nbas)]:
        fused = _np(fn(mol, b0, b1))
        monkeypatch.setattr(_eri, "FUSED_SPH", False)
        two = _np(fn(mol, b0, b1))
        monkeypatch.setattr(_eri, "FUSED_SPH", True)
        assert fused.shape == two.shape and not np.isnan(fused).any(), (b0, b1)
        assert np.abs(fused - two).max() <= 1e-12 * np.abs(two).max(), (b0, b1)
