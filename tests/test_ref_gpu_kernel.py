"""The ERI kernels against the reference's own kernels run on the same GPU.

oracle/_ref/libref_eri_gpu.so holds the reference's fill_int2e_kernel and
fill_int2e_ip1_kernel built for sm_100a (oracle/build_ref.py) and launched as
the reference launches them (ref: ccsd_gpu/cuda/int2e_gpu.py:39-108,
ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216).  Cartesian s2kl blocks of the
package must agree with them to the reference tests' bar: 1e-10 of the block
maximum plus 1e-12 (ref: tests/test_int2e_ip1_gpu.py uses atol 1e-10).
"""
import numpy as np
import pytest
import torch

from oracle import ref_gpu
from tests.test_oracle import block_close

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(), reason="reference GPU kernels not built")]


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("deriv", [0, 1])
def test_h2o_blocks_match_reference_gpu_kernel(deriv):
    from ccsd_gpu_b200 import compute_int2e_gpu, compute_int2e_ip1_gpu
    from ccsd_gpu_b200.gto import M
    mol = M(atom="O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587", basis="cc-pvdz", cart=True)
    rb = ref_gpu.RefBasis(mol, torch.device("cuda", 0))
    fn = compute_int2e_ip1_gpu if deriv else compute_int2e_gpu
    for b0, b1 in [(0, 1), (0, mol.nbas), (3, 5), (mol.nbas - 1, mol.nbas)]:
        ref = _np(ref_gpu.eri_cart(rb, b0, b1, deriv))
        got = _np(fn(mol, b0, b1))
        assert got.shape == ref.shape
        assert block_close(got, ref), (deriv, b0, b1, np.abs(got - ref).max())


def test_ethanol_atom_blocks_match_reference_gpu_kernel():
    """int2e_ip1 of every atom's shell block, as the reference's gradient loop
    requests them (ref: ccsd_gpu/gpu_ccsd_grad.py:449-457)."""
    from ccsd_gpu_b200 import compute_int2e_ip1_gpu, workloads
    from ccsd_gpu_b200.gto import M
    sym, xyz = workloads.ethanol_atoms(seed=0)
    mol = M(atom=workloads.atom_string(sym, xyz), basis="cc-pvdz", cart=True)
    rb = ref_gpu.RefBasis(mol, torch.device("cuda", 0))
    for a in (0, 2, 8):
        b0, b1 = (int(x) for x in mol.offset_nr_by_atom()[a][:2])
        ref = _np(ref_gpu.eri_cart(rb, b0, b1, 1))
        got = _np(compute_int2e_ip1_gpu(mol, b0, b1))
        assert block_close(got, ref), (a, np.abs(got - ref).max())
