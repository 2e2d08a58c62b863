"""Drop-in for ``ccsd_gpu.cuda.int2e_gpu`` (ref: ccsd_gpu/cuda/int2e_gpu.py:186-215).

``compute_int2e_gpu(mol, b0, b1)`` equals
``mol.intor('int2e', aosym='s2kl', shls_slice=(b0, b1, 0, nbas, 0, nbas, 0, nbas))``
reshaped to ``(nf, nao, nao_pair)``: ``[fi_local, fj_abs, k*(k+1)/2 + l]`` with
k >= l, in the molecule's native basis (Cartesian or spherical).  Returned as a
float64 CUDA ``torch.Tensor``.
"""
from ._eri import compute_s2kl
from .basis import _check_mol, get_basis_cached as _get_basis_cached  # noqa: F401


def compute_int2e_gpu(mol, b0, b1):
    return compute_s2kl(mol, b0, b1, 0)[0]
