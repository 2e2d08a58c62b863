"""Drop-in for ``ccsd_gpu.cuda.int2e_ip1_gpu`` (ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:296-326).

``compute_int2e_ip1_gpu(mol, b0, b1)`` equals
``mol.intor('int2e_ip1', comp=3, aosym='s2kl', shls_slice=(b0, b1, 0, nbas, 0, nbas, 0, nbas))``
reshaped to ``(3, nf, nao, nao_pair)``: component x, y, z of d/dr_1 on the
first function, PySCF sign convention.  Returned as a float64 CUDA tensor.
"""
from ._eri import compute_s2kl
from .basis import _check_mol, _basis_cache, decontract_bas as _decontract_bas  # noqa: F401
from .basis import get_basis_cached as _get_basis_cached  # noqa: F401


def compute_int2e_ip1_gpu(mol, b0, b1):
    return compute_s2kl(mol, b0, b1, 1)
