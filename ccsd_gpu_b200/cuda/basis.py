"""Geometry-independent basis topology, cached per (basis layout, device).

Mirrors ``_check_mol``, ``_decontract_bas`` and ``_get_basis_cached``
(ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:36-141): general contractions (nctr > 1)
are split into nctr = 1 shells that point at their own coefficient column, so
every device shell has (l+1)(l+2)/2 Cartesian functions.  Unlike the
reference no kl-pair list is stored: the kernels decode pair indices
arithmetically.  The sparse Cartesian->spherical factors used by the fused
transform are cached here too.
"""
import numpy as np
import torch

L_MAX = 4
ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, PTR_EXP, PTR_COEFF = 0, 1, 2, 3, 5, 6


def _check_mol(mol):
    """True iff every shell has l <= 4 (ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:36-40)."""
    return int(np.asarray(mol._bas)[:, ANG_OF].max()) <= L_MAX


def decontract_bas(bas):
    bas = np.asarray(bas, dtype=np.int32)
    rows, orig2dc = [], []
    for ish in range(len(bas)):
        nctr, nprim, pc = int(bas[ish, NCTR_OF]), int(bas[ish, NPRIM_OF]), int(bas[ish, PTR_COEFF])
        idx = []
        for c in range(nctr):
            r = bas[ish].copy()
            r[NCTR_OF] = 1
            r[PTR_COEFF] = pc + c * nprim
            idx.append(len(rows))
            rows.append(r)
        orig2dc.append(idx)
    dc = np.ascontiguousarray(np.array(rows, dtype=np.int32).reshape(-1, 8))
    l = dc[:, ANG_OF]
    ao_loc = np.zeros(len(dc) + 1, dtype=np.int32)
    np.cumsum((l + 1) * (l + 2) // 2, out=ao_loc[1:])
    return dc, ao_loc, orig2dc


def sparse_columns(C):
    """CSR-by-column of a dense (ncart, nsph) matrix: ptr, idx, val."""
    ptr = [0]
    idx, val = [], []
    for s in range(C.shape[1]):
        nz = np.nonzero(C[:, s])[0]
        idx.extend(nz.tolist())
        val.extend(C[nz, s].tolist())
        ptr.append(len(idx))
    return (np.asarray(ptr, dtype=np.int32), np.asarray(idx, dtype=np.int32),
            np.asarray(val, dtype=np.float64))


class BasisTopology:
    def __init__(self, mol, device):
        self.dc_bas, self.dc_ao_loc, self.orig2dc = decontract_bas(mol._bas)
        self.dc_nbas = len(self.dc_bas)
        self.nao_cart = int(self.dc_ao_loc[-1])
        self.lmax = int(self.dc_bas[:, ANG_OF].max())
        self.max_prim = int(self.dc_bas[:, NPRIM_OF].max())
        self.device = device
        self.bas_dev = torch.from_numpy(self.dc_bas).to(device)
        self.ao_loc_dev = torch.from_numpy(self.dc_ao_loc).to(device)
        self._sph = None
        self._sph_fused = None
        self._mol_bas = np.asarray(mol._bas).copy()
        self._sph_src = mol

    def sph(self):
        """Sparse cart->sph factors on the device (full matrix by column)."""
        if self._sph is None:
            C = np.asarray(self._sph_src.cart2sph_coeff())
            ptr, idx, val = sparse_columns(C)
            self._sph = dict(C=C,
                             ptr=torch.from_numpy(ptr).to(self.device),
                             idx=torch.from_numpy(idx).to(self.device),
                             val=torch.from_numpy(val).to(self.device),
                             ao_loc_sph=np.asarray(self._sph_src.ao_loc_nr(cart=False)),
                             ao_loc_cart=np.asarray(self._sph_src.ao_loc_nr(cart=True)))
            self._sph_src = None
        return self._sph

    def sph_fused(self):
        """(spherical AO offsets of the decontracted shells, d-shell cart->sph
        factors 5 x 6) on the device, for ccsd_b200_eri_s2kl_sph (l <= 2)."""
        if getattr(self, "_sph_fused", None) is None:
            s = self.sph()
            C = s["C"]
            l = self.dc_bas[:, ANG_OF].astype(np.int64)
            ls = np.zeros(len(l) + 1, dtype=np.int32)
            np.cumsum(2 * l + 1, out=ls[1:])
            c2s = np.zeros((5, 6))
            for d in range(len(l)):
                lc0, ls0, nc, ns = int(self.dc_ao_loc[d]), int(ls[d]), int((l[d] + 1) * (l[d] + 2) // 2), int(2 * l[d] + 1)
                blk = C[lc0:lc0 + nc, ls0:ls0 + ns]
                if l[d] < 2:
                    if not np.array_equal(blk, np.eye(nc)):
                        raise ValueError("cart2sph factors of an s or p shell are not the identity")
                elif l[d] == 2:
                    c2s = blk.T.copy()
            self._sph_fused = (torch.from_numpy(ls).to(self.device),
                               torch.from_numpy(np.ascontiguousarray(c2s)).to(self.device))
        return self._sph_fused

    def sph_block(self, b0, b1):
        """Sparse factors restricted to the i-shell block [b0, b1) (original shells)."""
        s = self.sph()
        lc, ls = s["ao_loc_cart"], s["ao_loc_sph"]
        Ci = s["C"][lc[b0]:lc[b1], ls[b0]:ls[b1]]
        ptr, idx, val = sparse_columns(Ci)
        return (torch.from_numpy(ptr).to(self.device), torch.from_numpy(idx).to(self.device),
                torch.from_numpy(val).to(self.device))


_basis_cache = {}


def get_basis_cached(mol, device=None):
    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    key = (np.asarray(mol._bas).tobytes(), bool(mol.cart), device.index)
    topo = _basis_cache.get(key)
    if topo is None:
        topo = BasisTopology(mol, device)
        _basis_cache[key] = topo
    return topo


def upload_geometry(mol, device):
    """_atm and _env change with the geometry; they are uploaded per call."""
    atm = torch.from_numpy(np.ascontiguousarray(mol._atm, dtype=np.int32)).to(device, non_blocking=False)
    env = torch.from_numpy(np.ascontiguousarray(mol._env, dtype=np.float64)).to(device, non_blocking=False)
    return atm, env
