"""Two-electron gradient term sum (d/dR_A ij|kl) Gamma[ijkl] without stored
ERI derivatives.

The reference computes int2e_ip1 for each atom's shell block, keeps the block
in memory and contracts it with the 2-RDM and the HF density products
(ref: ccsd_gpu/gpu_ccsd_grad.py:416-500).  Here one native call
(``ccsd_b200_eri_ip1_contract``) builds every (dI J|K L) shell quartet and
contracts it with Gamma inside the kernel; only three numbers per quartet
leave the SM, and a fixed-order segment sum turns them into per-atom values.
"""
from types import SimpleNamespace

import numpy as np
import torch

from .. import _native, tune
from .basis import _check_mol, get_basis_cached, upload_geometry


def _lclass(l, q):
    li, lj, lk, ll = (l[q[:, c]] for c in range(4))
    return ((li * 5 + lj) * 5 + lk) * 5 + ll


def gradient_quartets(topo, natm):
    """(quartets int32 (nq, 4) on the device, seg int64 (natm + 1,) on the device).

    Every (I, J, K >= L) quartet of decontracted shells, grouped by the atom
    of I (segment a = atom a), L-class ordered inside a segment.  Cached on the
    topology (the list depends only on the basis layout).
    """
    cache = topo.__dict__.setdefault("_grad_quartets", {})
    if natm in cache:
        return cache[natm]
    bas = topo.dc_bas
    nb = topo.dc_nbas
    atom = bas[:, 0].astype(np.int64)
    l = bas[:, 1].astype(np.int64)
    k, ll = np.tril_indices(nb)
    kl = np.stack([k, ll], 1)
    parts, seg = [], [0]
    for a in range(natm):
        ish = np.nonzero(atom == a)[0]
        if len(ish):
            ij = np.stack(np.meshgrid(ish, np.arange(nb), indexing="ij"), -1).reshape(-1, 2)
            q = np.concatenate([np.repeat(ij, len(kl), 0), np.tile(kl, (len(ij), 1))], 1)
            q = q[np.argsort(_lclass(l, q), kind="stable")]
            parts.append(q)
            seg.append(seg[-1] + len(q))
        else:
            seg.append(seg[-1])
    q = np.concatenate(parts, 0).astype(np.int32) if parts else np.zeros((0, 4), np.int32)
    out = (torch.from_numpy(np.ascontiguousarray(q)).to(topo.device),
           torch.tensor(seg, dtype=torch.int64, device=topo.device))
    cache[natm] = out
    return out


def gamma_to_cart(mol, gamma):
    """Back-transform a spherical-AO [nao]^4 density to the Cartesian AO basis
    of the decontracted shells (sum_p I_sph Gamma_sph = sum_a I_cart Gamma_cart)."""
    if mol.cart:
        return gamma
    topo = get_basis_cached(mol, gamma.device)
    T = torch.as_tensor(topo.sph()["C"], dtype=torch.float64, device=gamma.device)   # (ncart, nsph)
    g = torch.einsum("ap,pqrs->aqrs", T, gamma)
    g = torch.einsum("bq,aqrs->abrs", T, g)
    g = torch.einsum("cr,abrs->abcs", T, g)
    return torch.einsum("ds,abcs->abcd", T, g).contiguous()


def contract_int2e_ip1(mol, gamma, stream=None):
    """(natm, 3) FP64 tensor: out[A, x] = sum_{i on A, j, k, l} (d/dx_i ij|kl) gamma[ijkl].

    ``gamma``: (nao,)*4 FP64 on the GPU in the molecule's AO basis, symmetric
    in k <-> l.  Same sign convention as PySCF's int2e_ip1 (derivative of the
    bra function i with respect to its electron coordinate).
    """
    _native.require_cuda(gamma)
    if not _check_mol(mol):
        raise ValueError("shells with l > 4 are not supported (nroots > 9)")
    dev = gamma.device
    topo = get_basis_cached(mol, dev)
    gc = gamma_to_cart(mol, gamma.to(torch.float64))
    naoc = topo.nao_cart
    if tuple(gc.shape) != (naoc,) * 4:
        raise ValueError("gamma has shape %s, expected (%d,)*4" % (tuple(gamma.shape), mol.nao_nr()))
    atm, env = upload_geometry(mol, dev)
    q, seg = gradient_quartets(topo, mol.natm)
    nq = int(q.shape[0])
    if nq:
        ds = SimpleNamespace(atm=atm, bas=topo.bas_dev, env=env, lmax=topo.lmax)
        tune.tune_eri_heavy(ds, topo.dc_bas, q, 1, tune.basis_dshare(topo.dc_bas))
        tune.tune_eri_paths(ds, topo.dc_bas, q, 1, tune.basis_dshare(topo.dc_bas))
    qwork = torch.empty((max(nq, 1), 3), dtype=torch.float64, device=dev)
    out = torch.empty((mol.natm, 3), dtype=torch.float64, device=dev)
    _native.call("ccsd_b200_eri_ip1_contract", _native.ptr(atm), _native.ptr(topo.bas_dev), _native.ptr(env),
                 _native.ptr(topo.ao_loc_dev), naoc, _native.ptr(gc), _native.ptr(q), nq, _native.ptr(seg),
                 mol.natm, topo.lmax, _native.ptr(qwork), _native.ptr(out), _native.stream(stream))
    return out


def contract_int2e_ip1_rows(mol, rows, atom, stream=None):
    """(3,) FP64 tensor: sum_{i on atom, j, k, l} (d/dx_i ij|kl) gamma[ijkl] from
    only the atom's rows of gamma.

    ``rows``: (nrows, nao, nao, nao) FP64 on the GPU, the rows
    ``mol.offset_nr_by_atom()[atom][2:4]`` of gamma in the molecule's AO
    basis (symmetric in k <-> l).  The rows go to the Cartesian basis of the
    decontracted shells (the atom's rows only), and the atom's segment of the
    gradient quartet list is contracted with them by
    ``ccsd_b200_eri_ip1_contract_rows``.  Summed over atoms this equals
    :func:`contract_int2e_ip1` of the whole gamma, which never has to exist.
    """
    _native.require_cuda(rows)
    if not _check_mol(mol):
        raise ValueError("shells with l > 4 are not supported (nroots > 9)")
    dev = rows.device
    topo = get_basis_cached(mol, dev)
    naoc = topo.nao_cart
    s0, s1, p0, p1 = (int(x) for x in mol.offset_nr_by_atom()[atom])
    out = torch.zeros(3, dtype=torch.float64, device=dev)
    if s1 <= s0:
        return out
    d0, d1 = topo.orig2dc[s0][0], topo.orig2dc[s1 - 1][-1] + 1
    c0, c1 = int(topo.dc_ao_loc[d0]), int(topo.dc_ao_loc[d1])
    if tuple(rows.shape) != (p1 - p0,) + (mol.nao_nr(),) * 3:
        raise ValueError("rows has shape %s, expected (%d,) + (%d,)*3" % (tuple(rows.shape), p1 - p0, mol.nao_nr()))
    rows = rows.to(torch.float64)
    if not mol.cart:
        from ..lowmem import transform_rows
        T = torch.as_tensor(topo.sph()["C"], dtype=torch.float64, device=dev)      # (ncart, nsph)
        rows = transform_rows(rows.contiguous(), T[c0:c1, p0:p1].T, T.T, T.T, T.T).contiguous()
    atm, env = upload_geometry(mol, dev)
    q, seg = gradient_quartets(topo, mol.natm)
    segh = seg.cpu().numpy()
    qa = q[int(segh[atom]):int(segh[atom + 1])]
    nq = int(qa.shape[0])
    if nq:
        ds = SimpleNamespace(atm=atm, bas=topo.bas_dev, env=env, lmax=topo.lmax)
        tune.tune_eri_heavy(ds, topo.dc_bas, q, 1, tune.basis_dshare(topo.dc_bas))
        tune.tune_eri_paths(ds, topo.dc_bas, q, 1, tune.basis_dshare(topo.dc_bas))
    qwork = torch.empty((max(nq, 1), 3), dtype=torch.float64, device=dev)
    seg1 = torch.tensor([0, nq], dtype=torch.int64, device=dev)
    _native.call("ccsd_b200_eri_ip1_contract_rows", _native.ptr(atm), _native.ptr(topo.bas_dev), _native.ptr(env),
                 _native.ptr(topo.ao_loc_dev), naoc, _native.ptr(rows), c0, c1 - c0, _native.ptr(qa), nq,
                 _native.ptr(seg1), 1, topo.lmax, _native.ptr(qwork), _native.ptr(out.view(1, 3)),
                 _native.stream(stream))
    return out
