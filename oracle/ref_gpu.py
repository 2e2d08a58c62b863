"""ORACLE / COMPARATOR -- test and benchmark infrastructure only.

Python binding of oracle/_ref/libref_eri_gpu.so (built from
oracle/ref_eri_gpu.cu by oracle/build_ref.py): the reference's own
fill_int2e_kernel / fill_int2e_ip1_kernel (ref: ccsd_gpu/cuda/int2e_module.py:130-463,
ccsd_gpu/cuda/int2e_ip1_module.py:273-667) compiled for sm_100a and launched
the way the reference's _compute_cart launches them: one launch per
decontracted i-shell over every (j, k >= l) shell triple
(ref: ccsd_gpu/cuda/int2e_gpu.py:39-108, ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216).

It serves two purposes only: a GPU-side parity check of the package's ERI
kernels against the reference's kernels, and the reference-GPU timing beside
them (``bench.py --workload refgpu``).  The package never imports this module.
"""
import ctypes
import os

import numpy as np
import torch

LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_eri_gpu.so")
_lib = None


def available():
    return os.path.exists(LIB)


def _load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("%s is not built (python oracle/build_ref.py <reference checkout>)" % LIB)
        lib = ctypes.CDLL(LIB)
        vp, ci = ctypes.c_void_p, ctypes.c_int
        lib.ref_gpu_eri_cart.restype = ci
        lib.ref_gpu_eri_cart.argtypes = [ci, vp, vp, vp, vp, vp, vp, vp, ci, ci, ci, ci, vp, ci, ci, ci, vp]
        _lib = lib
    return _lib


class RefBasis:
    """Decontracted basis of ``mol`` as the reference's _get_basis_cached
    builds it (ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:88-141): the package's own
    decontraction (the same rule), the (k >= l) pair list in row order, and
    device copies of atm, bas, env, ao_loc."""

    def __init__(self, mol, device):
        from ccsd_gpu_b200.cuda.basis import decontract_bas
        self.dc_bas, self.dc_ao_loc, self.orig2dc = decontract_bas(np.asarray(mol._bas))
        self.dc_bas = np.ascontiguousarray(self.dc_bas, dtype=np.int32)
        self.dc_ao_loc = np.ascontiguousarray(self.dc_ao_loc, dtype=np.int32)
        self.nbas = len(self.dc_bas)
        self.nao = int(self.dc_ao_loc[-1])
        k, l = np.tril_indices(self.nbas)
        self.kl = np.ascontiguousarray(np.stack([k, l], 1).astype(np.int32).ravel())
        self.n_kl = len(k)
        self.max_l = int(self.dc_bas[:, 1].max())
        self.max_prim = int(self.dc_bas[:, 2].max())
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.atm = t(np.asarray(mol._atm, dtype=np.int32))
        self.env = t(np.asarray(mol._env, dtype=np.float64))
        self.bas_dev = t(self.dc_bas)
        self.ao_loc_dev = t(self.dc_ao_loc)
        self.kl_dev = t(self.kl)

    def dc_range(self, b0, b1):
        return self.orig2dc[b0][0], self.orig2dc[b1 - 1][-1] + 1


def eri_cart(rb, b0, b1, deriv, out=None, stream=None):
    """Cartesian s2kl block ((3 if deriv) x nf x nao x nao(nao+1)/2) of the
    original shells [b0, b1) from the reference's kernels, as a CUDA tensor."""
    d0, d1 = rb.dc_range(b0, b1)
    nf = int(rb.dc_ao_loc[d1] - rb.dc_ao_loc[d0])
    npair = rb.nao * (rb.nao + 1) // 2
    shape = ((3,) if deriv else (1,)) + (nf, rb.nao, npair)
    if out is None:
        out = torch.empty(shape, dtype=torch.float64, device=rb.atm.device)
    st = stream if stream is not None else torch.cuda.current_stream(rb.atm.device).cuda_stream
    rc = _load().ref_gpu_eri_cart(int(deriv), out.data_ptr(), rb.atm.data_ptr(), rb.bas_dev.data_ptr(),
                                  rb.env.data_ptr(), rb.ao_loc_dev.data_ptr(),
                                  rb.dc_bas.ctypes.data, rb.dc_ao_loc.ctypes.data, d0, d1, rb.nbas, rb.nao,
                                  rb.kl_dev.data_ptr(), rb.n_kl, rb.max_l, rb.max_prim, ctypes.c_void_p(st))
    if rc != 0:
        raise RuntimeError("ref_gpu_eri_cart failed: CUDA error %d" % rc)
    return out if deriv else out[0]
