"""Fused int2e_ip1 . Gamma kernel (derivative integrals never stored) against
the oracle's dense int2e_ip1 tensor contracted on the host."""
import numpy as np
import pytest
import torch

from oracle import scf_cc_oracle as Q

pytestmark = pytest.mark.gpu


def _gamma(n, seed):
    g = np.random.default_rng(seed).standard_normal((n, n, n, n))
    return 0.5 * (g + g.transpose(0, 1, 3, 2))          # symmetric in k <-> l only


@pytest.mark.parametrize("cart", [False, True])
def test_ip1_gamma_contraction_matches_oracle(cart):
    from ccsd_gpu_b200.cuda.ip1_contract import contract_int2e_ip1
    from ccsd_gpu_b200.gto import M
    mol = M(atom="O 0 0 0; H 0 -0.757 0.587; H 0.05 0.757 0.587", basis="cc-pvdz", cart=cart)
    n = mol.nao_nr()
    gam = _gamma(n, 11)
    I = Q.full_eri_ip1(mol)                                  # (3, n, n, n, n), derivative on i
    per_ao = np.einsum("xijkl,ijkl->ix", I, gam)
    off = mol.offset_nr_by_atom()
    ref = np.array([per_ao[off[a][2]:off[a][3]].sum(0) for a in range(mol.natm)])
    got = contract_int2e_ip1(mol, torch.from_numpy(gam).cuda()).cpu().numpy()
    scale = np.abs(np.einsum("xijkl,ijkl->ix", np.abs(I), np.abs(gam))).max()
    assert np.abs(got - ref).max() <= 1e-12 * scale, (got, ref)


def test_ip1_gamma_contraction_is_deterministic_and_translation_invariant():
    """Bit-identical on repeat; with a gamma symmetric in (ij), (kl) and
    (ij) <-> (kl), the per-atom sums add up to zero (translation invariance)."""
    from ccsd_gpu_b200.cuda.ip1_contract import contract_int2e_ip1
    from ccsd_gpu_b200.gto import M
    mol = M(atom="C 0 0 0; O 0 0 1.2; H 0.9 0 -0.5; H -0.9 0 -0.5", basis="cc-pvdz")
    n = mol.nao_nr()
    g = np.random.default_rng(3).standard_normal((n, n, n, n))
    g = g + g.transpose(1, 0, 2, 3)
    g = g + g.transpose(0, 1, 3, 2)
    g = g + g.transpose(2, 3, 0, 1)
    gt = torch.from_numpy(g).cuda()
    a = contract_int2e_ip1(mol, gt)
    b = contract_int2e_ip1(mol, gt)
    assert torch.equal(a, b)
    tot = a.sum(0).abs().max().item()
    assert tot <= 1e-10 * a.abs().max().item()
