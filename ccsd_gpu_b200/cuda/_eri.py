"""Shared host logic of the int2e / int2e_ip1 drop-in entry points."""
import numpy as np
import torch

from .. import _native
from .basis import _check_mol, get_basis_cached, upload_geometry


# Cartesian functions per quartet above which the CTA kernel is used: int2e,
# int2e_ip1 (the same thresholds as heavy_nf() in csrc/eri.cu)
HEAVY_NF = {0: 1000, 1: 500}

# spherical blocks of l <= 2 bases in one pass (ccsd_b200_eri_s2kl_sph);
# False: Cartesian kernel + separate sparse transform (the l > 2 route)
FUSED_SPH = True


def heavy_quartets(topo, d0, d1, deriv=0):
    """(n, 4) int32 device list of the block's quartets with more than HEAVY_NF[deriv] functions."""
    cache = topo.__dict__.setdefault("_heavy", {})
    if (d0, d1, deriv) in cache:
        return cache[(d0, d1, deriv)]
    l = topo.dc_bas[:, 1].astype(np.int64)
    nc = (l + 1) * (l + 2) // 2
    nb = topo.dc_nbas
    k, ll = np.tril_indices(nb)
    nkl = nc[k] * nc[ll]
    i = np.arange(d0, d1)
    j = np.arange(nb)
    nij = (nc[i][:, None] * nc[j][None, :]).ravel()
    ij, pp = np.nonzero(nij[:, None] * nkl[None, :] > HEAVY_NF[deriv])
    q = np.stack([i[ij // nb], j[ij % nb], k[pp], ll[pp]], 1).astype(np.int32)
    order = np.argsort(-(nij[ij] * nkl[pp]), kind="stable")     # heaviest first
    dev = torch.from_numpy(np.ascontiguousarray(q[order]).reshape(-1, 4)).to(topo.device)
    cache[(d0, d1, deriv)] = dev
    return dev


def compute_s2kl(mol, b0, b1, deriv, stream=None):
    """s2kl block (ncomp, nf, nao, nao_pair) in the molecule's native basis."""
    _native.require_cuda()
    if not (0 <= b0 < b1 <= mol.nbas):
        raise ValueError("invalid shell range [%d, %d) for nbas = %d" % (b0, b1, mol.nbas))
    if not _check_mol(mol):
        raise ValueError("shells with l > 4 are not supported (nroots > 9)")
    dev = torch.device("cuda", torch.cuda.current_device())
    topo = get_basis_cached(mol, dev)
    atm, env = upload_geometry(mol, dev)
    d0, d1 = topo.orig2dc[b0][0], topo.orig2dc[b1 - 1][-1] + 1
    loc = topo.dc_ao_loc
    nfc = int(loc[d1] - loc[d0])
    naoc = topo.nao_cart
    npc = naoc * (naoc + 1) // 2
    ncomp = 3 if deriv else 1
    st = _native.stream(stream)
    hq = heavy_quartets(topo, d0, d1, int(deriv))
    if not mol.cart and topo.lmax <= 2 and FUSED_SPH:
        # one pass: each quartet's block is transformed to spherical
        # functions in the kernel that computes it
        ls_dev, c2s = topo.sph_fused()
        ls = topo.sph()["ao_loc_sph"]
        nfs = int(ls[b1] - ls[b0])
        naos = int(ls[-1])
        out = torch.empty((ncomp, nfs, naos, naos * (naos + 1) // 2), dtype=torch.float64, device=dev)
        _native.call("ccsd_b200_eri_s2kl_sph", int(deriv), _native.ptr(atm), _native.ptr(topo.bas_dev),
                     _native.ptr(env), topo.dc_nbas, _native.ptr(topo.ao_loc_dev), _native.ptr(ls_dev),
                     _native.ptr(c2s), d0, d1, naos, topo.lmax, _native.ptr(hq), int(hq.shape[0]), _native.ptr(out),
                     st)
        return out
    cart = torch.empty((ncomp, nfc, naoc, npc), dtype=torch.float64, device=dev)
    _native.call("ccsd_b200_eri_s2kl_cart", int(deriv), _native.ptr(atm), _native.ptr(topo.bas_dev),
                 _native.ptr(env), topo.dc_nbas, _native.ptr(topo.ao_loc_dev), d0, d1, naoc, topo.lmax,
                 _native.ptr(hq), int(hq.shape[0]), _native.ptr(cart), st)
    if mol.cart:
        return cart
    sph = topo.sph()
    ls = sph["ao_loc_sph"]
    nfs = int(ls[b1] - ls[b0])
    naos = int(ls[-1])
    ptr_i, idx_i, val_i = topo.sph_block(b0, b1)
    tmp = torch.empty((ncomp, nfs, naos, npc), dtype=torch.float64, device=dev)
    out = torch.empty((ncomp, nfs, naos, naos * (naos + 1) // 2), dtype=torch.float64, device=dev)
    _native.call("ccsd_b200_cart2sph_s2kl", _native.ptr(cart), _native.ptr(tmp), _native.ptr(out),
                 ncomp, nfc, naoc, nfs, naos, _native.ptr(ptr_i), _native.ptr(idx_i), _native.ptr(val_i),
                 _native.ptr(sph["ptr"]), _native.ptr(sph["idx"]), _native.ptr(sph["val"]), st)
    # tmp/cart go back to torch's stream-ordered caching allocator: safe to drop here
    return out
