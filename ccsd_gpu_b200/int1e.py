"""One-electron integrals on the GPU, PySCF names and conventions.

``intor1e(mol, name, origin_atom=None)`` returns a float64 CUDA tensor of shape
(nao, nao) or (3, nao, nao) in the molecule's native basis, equal to
``mol.intor(name)`` for the names below (libcint's "ip" forms put d/dr on the
first function):

  int1e_ovlp, int1e_kin, int1e_nuc, int1e_rinv (origin at an atom),
  int1e_ipovlp, int1e_ipkin, int1e_ipnuc, int1e_iprinv.

These are what the gradient's one-electron terms read through PySCF
(ref: ccsd_gpu/gpu_ccsd_grad.py:554-584: hcore_generator, get_ovlp).
"""
import numpy as np
import torch

from . import _native
from .cuda.basis import get_basis_cached, upload_geometry

OPS = {"int1e_ovlp": 0, "int1e_kin": 1, "int1e_nuc": 2, "int1e_rinv": 3,
       "int1e_ipovlp": 4, "int1e_ipkin": 5, "int1e_ipnuc": 6, "int1e_iprinv": 7}


def intor1e(mol, name, origin_atom=None):
    _native.require_cuda()
    op = OPS[name]
    dev = torch.device("cuda", torch.cuda.current_device())
    topo = get_basis_cached(mol, dev)
    atm, env = upload_geometry(mol, dev)
    naoc = topo.nao_cart
    ncomp = 3 if op >= 4 else 1
    out = torch.empty((ncomp, naoc, naoc), dtype=torch.float64, device=dev)
    org = -1 if origin_atom is None else int(origin_atom)
    if op in (3, 7) and org < 0:
        raise ValueError("%s needs origin_atom" % name)
    _native.call("ccsd_b200_int1e_cart", op, _native.ptr(atm), mol.natm, _native.ptr(topo.bas_dev), topo.dc_nbas,
                 _native.ptr(env), _native.ptr(topo.ao_loc_dev), topo.lmax, org, _native.ptr(out), _native.stream())
    if not mol.cart:
        C = _c2s_dense(topo, mol, dev)
        out = torch.einsum("pi,xpq,qj->xij", C, out, C)
    return out if ncomp == 3 else out[0]


def _c2s_dense(topo, mol, dev):
    c = topo.__dict__.get("_c2s_dense")
    if c is None:
        c = torch.from_numpy(np.asarray(mol.cart2sph_coeff())).to(dev)
        topo._c2s_dense = c
    return c
