"""Explicit shell-quartet lists: integrals consumed in-kernel (checksums), Schwarz bounds.

This is the batched entry the ERI throughput benchmark and the full-size
parity checks use; the reference has no counterpart (it only materialises
s2kl blocks, ref: ccsd_gpu/cuda/int2e_gpu.py:186-215).
"""
import numpy as np
import torch

from .. import _native


class DeviceShells:
    """_atm/_bas/_env of decontracted shells resident on the device."""

    def __init__(self, shells, device=None):
        _native.require_cuda()
        device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        bas = np.asarray(shells._bas, dtype=np.int32)
        if (bas[:, 3] != 1).any():
            raise ValueError("quartet entry points take decontracted shells (nctr == 1)")
        self.atm = torch.from_numpy(np.ascontiguousarray(shells._atm, dtype=np.int32)).to(device)
        self.bas = torch.from_numpy(np.ascontiguousarray(bas)).to(device)
        self.env = torch.from_numpy(np.ascontiguousarray(shells._env, dtype=np.float64)).to(device)
        self.lmax = int(bas[:, 1].max())
        if self.lmax > 4:
            raise ValueError("shells with l > 4 are not supported")
        self.nbas = len(bas)
        self.device = device


def quartet_checksums(ds, quartets, deriv, out=None, stream=None):
    """(nq, ncomp, 2) float64 checksums of the integrals of each quartet."""
    if quartets.dtype != torch.int32 or not quartets.is_cuda or quartets.dim() != 2 or quartets.shape[1] != 4:
        raise ValueError("quartets must be a (nq, 4) int32 CUDA tensor")
    quartets = quartets.contiguous()
    nq = quartets.shape[0]
    ncomp = 3 if deriv else 1
    if out is None:
        out = torch.empty((nq, ncomp, 2), dtype=torch.float64, device=quartets.device)
    _native.call("ccsd_b200_eri_quartet_checksums", int(deriv), _native.ptr(ds.atm), _native.ptr(ds.bas),
                 _native.ptr(ds.env), _native.ptr(quartets), nq, ds.lmax, _native.ptr(out), _native.stream(stream))
    return out


def schwarz_bounds(ds, pairs):
    """Q_ij >= sqrt(max |(ij|ij)|) for an (m, 2) array of shell pairs (Frobenius bound)."""
    p = np.asarray(pairs, dtype=np.int32)
    q = torch.from_numpy(np.ascontiguousarray(np.concatenate([p, p], 1))).to(ds.device)
    s = quartet_checksums(ds, q, 0)
    return torch.sqrt(torch.sqrt(s[:, 0, 1].clamp_min(0))).cpu().numpy()
