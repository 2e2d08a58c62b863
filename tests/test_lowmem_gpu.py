"""Bounded-memory paths (lowmem): blocked four-index transforms, the SCF without
the cached G, the ao2mo that writes only the MO blocks, and the gradient whose
two-electron density is built atom block by atom block (the reference streams
its gradient by shell blocks sized from max_memory,
ref: ccsd_gpu/gpu_ccsd_grad.py:416-432).  On small molecules the forced lean
path must reproduce the dense one; a (H2O)12/cc-pVDZ gradient (nao 288: every
dense (nao,)*4 FP64 tensor is 55 GB) must run through on one GPU."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _gradient(mol, precision):
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.scf import RHF
    mf = RHF(mol).run()
    cc = CCSD(mf, precision=precision)
    cc.kernel()
    cc.conv_tol_normt = 1e-9
    return mf.e_tot, cc.e_tot, cc.nuc_grad_method().kernel()


@pytest.mark.parametrize("precision", ["fp64", "tf32x3"])
def test_lean_gradient_matches_dense(precision):
    from ccsd_gpu_b200 import lowmem, workloads
    from ccsd_gpu_b200.contract import clear_pack_cache
    from ccsd_gpu_b200.gto import M
    sym, xyz = workloads.water_cluster_atoms(2, np.random.default_rng(3))
    mol = M(atom=workloads.atom_string(sym, xyz), basis="cc-pvdz")
    try:
        lowmem.force(False)
        e_hf, e_cc, g_dense = _gradient(mol, precision)
        clear_pack_cache()
        lowmem.force(True)
        e_hf2, e_cc2, g_lean = _gradient(mol, precision)
    finally:
        lowmem.force(None)
        clear_pack_cache()
    assert abs(e_hf - e_hf2) < 1e-9
    assert abs(e_cc - e_cc2) < (1e-9 if precision == "fp64" else 1e-7)
    assert np.abs(g_dense - g_lean).max() < (1e-9 if precision == "fp64" else 1e-7)


def test_blocked_transforms_match_einsum():
    from ccsd_gpu_b200 import lowmem
    g = torch.Generator(device="cuda").manual_seed(0)
    T = torch.randn((13,) * 4, dtype=torch.float64, device="cuda", generator=g)
    C = torch.randn((13, 11), dtype=torch.float64, device="cuda", generator=g)
    ref = torch.einsum("abcd,ap,bq,cr,ds->pqrs", T, C, C, C, C)
    assert (lowmem.transform_all(T, C, block=4) - ref).abs().max() < 1e-11 * ref.abs().max()
    rows = lowmem.transform_cols1(T, C, C[:, 3:7], C, C)
    assert (rows - ref[:, 3:7].transpose(0, 1)).abs().max() < 1e-11 * ref.abs().max()
    D = torch.randn((13, 13), dtype=torch.float64, device="cuda", generator=g)
    J, K = lowmem.jk_blocked(T, D, block=5)
    assert (J - torch.einsum("pqrs,rs->pq", T, D)).abs().max() < 1e-11 * J.abs().max()
    assert (K - torch.einsum("prqs,rs->pq", T, D)).abs().max() < 1e-11 * K.abs().max()


def test_gradient_nao_288_runs_in_bounded_memory():
    """(H2O)12/cc-pVDZ, nao 288: the dense chain would need about five
    (nao,)*4 tensors (275 GB); the lean paths keep at most two."""
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.contract import clear_pack_cache
    from ccsd_gpu_b200.gto import M
    sym, xyz = workloads.water_cluster_atoms(12, np.random.default_rng(0))
    mol = M(atom=workloads.atom_string(sym, xyz), basis="cc-pvdz")
    assert mol.nao_nr() == 288
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats()
    e_hf, e_cc, g = _gradient(mol, "tf32x3")
    peak = torch.cuda.max_memory_allocated()
    clear_pack_cache()
    torch.cuda.empty_cache()
    assert np.isfinite(g).all() and np.isfinite(e_cc)
    assert e_cc < e_hf
    # translational invariance of the analytic gradient
    assert np.abs(g.sum(0)).max() < 1e-5
    # the dense chain would hold about five (nao,)*4 tensors (275 GB)
    assert peak < torch.cuda.get_device_properties(0).total_memory
    print("nao 288 gradient: peak device memory %.1f GB" % (peak / 1e9))
