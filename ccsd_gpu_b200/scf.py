"""Closed-shell Hartree-Fock on the GPU (the SCF the reference runs in PySCF on
the CPU, examples/h2o_ccsd_grad.py:118-121).

ERIs come from :func:`full_eri_gpu` (each unique shell quartet computed once)
and stay resident as a dense (nao,)*4 FP64 tensor ((H2O)6/cc-pVDZ, nao = 144:
3.4 GB; nao = 288: 55 GB).  J/K, DIIS and the
eigen-solves are FP64 on the device.  The object exposes the attributes the
CCSD gradient reads from a PySCF RHF: mol, mo_energy, mo_coeff, mo_occ, e_tot,
make_rdm1, get_ovlp, get_hcore, get_veff, energy_nuc.
"""
from types import SimpleNamespace

import numpy as np
import torch

from . import _native, lowmem, tune
from .cuda.basis import _check_mol, get_basis_cached, upload_geometry
from .int1e import intor1e


def unique_quartets(topo):
    """int32 (nq, 4) device list of the unique decontracted-shell quartets
    (I >= J, K >= L, pair(IJ) >= pair(KL)), L-class ordered; cached."""
    q = topo.__dict__.get("_unique_quartets")
    if q is None:
        nb = topo.dc_nbas
        i, j = np.tril_indices(nb)
        P, Q = np.tril_indices(len(i))
        quart = np.stack([i[P], j[P], i[Q], j[Q]], 1).astype(np.int32)
        l = topo.dc_bas[:, 1].astype(np.int64)[quart]
        key = ((l[:, 0] * 5 + l[:, 1]) * 5 + l[:, 2]) * 5 + l[:, 3]
        quart = quart[np.argsort(key, kind="stable")]
        q = torch.from_numpy(np.ascontiguousarray(quart)).to(topo.device)
        topo._unique_quartets = q
    return q


def full_eri_gpu(mol):
    """(nao,)*4 chemist-notation ERI tensor on the GPU, native basis.

    Each unique shell quartet is computed once (``ccsd_b200_eri_full_cart``
    writes all eight index orders); a spherical basis is reached by four
    dense transforms of the Cartesian tensor."""
    _native.require_cuda()
    if not _check_mol(mol):
        raise ValueError("shells with l > 4 are not supported (nroots > 9)")
    dev = torch.device("cuda", torch.cuda.current_device())
    topo = get_basis_cached(mol, dev)
    atm, env = upload_geometry(mol, dev)
    q = unique_quartets(topo)
    n = topo.nao_cart
    ds = SimpleNamespace(atm=atm, bas=topo.bas_dev, env=env, lmax=topo.lmax)
    tune.tune_eri_heavy(ds, topo.dc_bas, q, 0, tune.basis_dshare(topo.dc_bas))
    tune.tune_eri_paths(ds, topo.dc_bas, q, 0, tune.basis_dshare(topo.dc_bas))
    g = torch.empty((n, n, n, n), dtype=torch.float64, device=dev)
    _native.call("ccsd_b200_eri_full_cart", _native.ptr(atm), _native.ptr(topo.bas_dev), _native.ptr(env),
                 _native.ptr(topo.ao_loc_dev), n, _native.ptr(q), int(q.shape[0]), topo.lmax, _native.ptr(g),
                 _native.stream())
    if mol.cart:
        return g
    T = torch.as_tensor(topo.sph()["C"], dtype=torch.float64, device=dev)      # (ncart, nsph)
    # blocked over the first spherical index: only the Cartesian tensor, the
    # spherical one and one block are live
    return lowmem.transform_all(g, T)


class RHF:
    """Restricted closed-shell SCF; ``kernel()`` returns the total energy."""

    def __init__(self, mol, conv_tol=1e-11, max_cycle=100, diis_space=8):
        _native.require_cuda()
        self.mol = mol
        self.conv_tol = conv_tol
        self.max_cycle = max_cycle
        self.diis_space = diis_space
        self.converged = False
        self._eri = None

    # -- integrals -----------------------------------------------------------
    @property
    def eri(self):
        if self._eri is None:
            self._eri = full_eri_gpu(self.mol)
        return self._eri

    def get_ovlp(self, mol=None):
        if getattr(self, "_S", None) is None:
            self._S = intor1e(self.mol, "int1e_ovlp")
        return self._S

    def get_hcore(self, mol=None):
        if getattr(self, "_h", None) is None:
            self._h = intor1e(self.mol, "int1e_kin") + intor1e(self.mol, "int1e_nuc")
        return self._h

    def get_jk(self, mol=None, dm=None):
        dm = torch.as_tensor(dm, dtype=torch.float64, device=self.eri.device)
        return lowmem.jk_blocked(self.eri, dm)

    def _coulomb_exchange(self):
        """G[pq, rs] = (pq|rs) - 1/2 (pr|qs) as an (n^2, n^2) matrix, built once
        per geometry: each Fock build is then one matrix-vector product that
        streams G at HBM bandwidth instead of a strided exchange contraction.
        None when a second (n,)*4 tensor would crowd out the later stages (the
        ao2mo and the gradient need about three more): J/K then come from the
        ERIs directly (lowmem.jk_blocked)."""
        if getattr(self, "_G", None) is None and not getattr(self, "_no_G", False):
            e = self.eri
            n = e.shape[0]
            if lowmem.lean(3, n, e.device):
                self._no_G = True
                return None
            g = e.clone()
            g.sub_(e.permute(0, 2, 1, 3), alpha=0.5)
            self._G = g.view(n * n, n * n)
        return getattr(self, "_G", None)

    def get_veff(self, mol=None, dm=None):
        dm = torch.as_tensor(dm, dtype=torch.float64, device=self.eri.device)
        n = dm.shape[0]
        G = self._coulomb_exchange()
        if G is None:
            J, K = lowmem.jk_blocked(self.eri, dm)
            return J - 0.5 * K
        return (G @ dm.reshape(n * n)).view(n, n)

    def energy_nuc(self):
        return self.mol.energy_nuc()

    def make_rdm1(self, mo_coeff=None, mo_occ=None):
        mo_coeff = self.mo_coeff if mo_coeff is None else mo_coeff
        mo_occ = self.mo_occ if mo_occ is None else mo_occ
        c = torch.as_tensor(mo_coeff, device=self.eri.device)
        o = torch.as_tensor(mo_occ, device=self.eri.device, dtype=torch.float64)
        return (c * o) @ c.T

    # -- SCF -----------------------------------------------------------------------
    def kernel(self):
        S, h = self.get_ovlp(), self.get_hcore()
        nocc = self.mol.nelectron // 2
        w, U = torch.linalg.eigh(S)
        X = U / torch.sqrt(w)
        e, Cp = torch.linalg.eigh(X.T @ h @ X)
        C = X @ Cp
        dm = 2 * C[:, :nocc] @ C[:, :nocc].T
        fs, errs = [], []
        e_old = 0.0
        F = h + self.get_veff(dm=dm)
        for it in range(self.max_cycle):
            err = F @ dm @ S - S @ dm @ F
            fs.append(F)
            errs.append(err)
            fs, errs = fs[-self.diis_space:], errs[-self.diis_space:]
            n = len(fs)
            if n > 1:
                E = torch.stack([x.reshape(-1) for x in errs])
                B = -torch.ones((n + 1, n + 1), dtype=torch.float64, device=S.device)
                B[n, n] = 0
                B[:n, :n] = E @ E.T
                rhs = torch.zeros(n + 1, dtype=torch.float64, device=S.device)
                rhs[n] = -1
                c = torch.linalg.solve(B, rhs)[:n]
                F = (c[:, None, None] * torch.stack(fs)).sum(0)
            e, Cp = torch.linalg.eigh(X.T @ F @ X)
            C = X @ Cp
            dm_new = 2 * C[:, :nocc] @ C[:, :nocc].T
            Fn = h + self.get_veff(dm=dm_new)
            etot = float(0.5 * (dm_new * (h + Fn)).sum()) + self.energy_nuc()
            done = abs(etot - e_old) < self.conv_tol and float((dm_new - dm).abs().max()) < 1e-8
            dm, e_old, F = dm_new, etot, Fn
            if done:
                break
        e, Cp = torch.linalg.eigh(X.T @ F @ X)
        self.mo_energy_t, self.mo_coeff_t = e, X @ Cp
        self.mo_energy = e.cpu().numpy()
        self.mo_coeff = self.mo_coeff_t.cpu().numpy()
        self.mo_occ = np.zeros(len(self.mo_energy))
        self.mo_occ[:nocc] = 2
        self.e_tot = etot
        self.converged = done
        return etot

    def run(self):
        self.kernel()
        return self

    def nuc_grad_method(self):
        return _GradNuc(self.mol)


class _GradNuc:
    def __init__(self, mol):
        self.mol = mol

    def grad_nuc(self):
        return self.mol.grad_nuc()
