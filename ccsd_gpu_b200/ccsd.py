"""Closed-shell CCSD on the GPU: AO->MO transform, T-amplitude solve, and the
hooks the gradient needs (a PySCF-like CCSD object).

The reference obtains T amplitudes from gpu4pyscf or PySCF
(examples/h2o_ccsd_grad.py:128-147); here the RCCSD amplitude equations (the
form of PySCF's rccsd.update_amps / rintermediates) run through the same
contraction engine as the Lambda solver, so ``precision`` ("fp64", "tf32x3",
"bf16x3") applies to both.  Energies, norms, denominators and DIIS are FP64.
Wvvvv is never formed: its ovvv*t1 parts are folded into o^3 v intermediates
and the bare (ac|bd) term is one contraction with tau.
"""
from types import SimpleNamespace

import numpy as np
import torch

from . import _native, lowmem
from .contract import check_status, contract, effective_mode
from .graphs import StepGraph, graph_cache_ok, solve_step

_T_CONSTS = ("fock", "mo_energy", "ovov", "ovvv", "ovoo", "ovvo", "oovv", "oooo", "vvvv")
from .gpu_ccsd_lambda import DIIS, DeviceEris, amplitude_norm_sq, host_copy, remember_device, solve_lambda_gpu


def ao2mo_gpu(mf, mo_coeff=None, frozen=0):
    """Chemist-notation MO blocks (PySCF ``_ChemistsERIs`` layout) on the GPU, FP64.

    ``frozen`` lowest orbitals are left out of the correlation space: the blocks
    and the Fock matrix span the active orbitals only, the Fock matrix still
    built from the full HF density."""
    C = torch.as_tensor(mf.mo_coeff if mo_coeff is None else mo_coeff, dtype=torch.float64,
                        device=mf.eri.device)
    nocc_all = int((np.asarray(mf.mo_occ) > 0).sum())
    dm = 2 * C[:, :nocc_all] @ C[:, :nocc_all].T
    C = C[:, frozen:]
    nocc = nocc_all - frozen
    fock = C.T @ (mf.get_hcore() + mf.get_veff(dm=dm)) @ C
    o, v = slice(0, nocc), slice(nocc, C.shape[1])
    if lowmem.lean(4, C.shape[0], C.device):
        blocks = _mo_blocks_lean(mf.eri, C, nocc)
        # the CC solves never read the AO ERIs: release them (and the SCF's
        # cached G) for the solves; mf.eri recomputes them when the gradient
        # asks (the AO ERIs are the largest tensor of the chain)
        if hasattr(mf, "_eri"):
            mf._eri = None
            mf._G = None
            torch.cuda.empty_cache()
    else:
        g = torch.einsum("pqrs,pi->iqrs", mf.eri, C)
        g = torch.einsum("iqrs,qj->ijrs", g, C)
        g = torch.einsum("ijrs,rk->ijks", g, C)
        g = torch.einsum("ijks,sl->ijkl", g, C)
        blocks = dict(oooo=g[o, o, o, o].contiguous(), ovoo=g[o, v, o, o].contiguous(),
                      ovvo=g[o, v, v, o].contiguous(), oovv=g[o, o, v, v].contiguous(),
                      ovov=g[o, v, o, v].contiguous(), ovvv=g[o, v, v, v].contiguous(),
                      vvvv=g[v, v, v, v].contiguous())
        del g
    e = SimpleNamespace(fock=fock, mo_energy=torch.diagonal(fock).clone(), **blocks)
    return DeviceEris(e)


def _mo_blocks_lean(eri, C, nocc):
    """The seven MO blocks without the (nmo,)*4 tensor: the rows with an
    occupied first index (nocc x nmo^3) and the vvvv rows, each built block by
    block from the AO ERIs (lowmem.transform_rows), so only the AO ERIs, the
    blocks and one row block are live."""
    nmo = C.shape[1]
    nvir = nmo - nocc
    bs = lowmem.block_size(max(C.shape[0], nmo))
    go = torch.empty((nocc, nmo, nmo, nmo), dtype=C.dtype, device=C.device)
    for i0 in range(0, nocc, bs):
        i1 = min(nocc, i0 + bs)
        go[i0:i1] = lowmem.transform_rows(eri, C[:, i0:i1], C, C, C)
    o, v = slice(0, nocc), slice(nocc, nmo)
    out = dict(oooo=go[:, o, o, o].contiguous(), ovoo=go[:, v, o, o].contiguous(), ovvo=go[:, v, v, o].contiguous(),
               oovv=go[:, o, v, v].contiguous(), ovov=go[:, v, o, v].contiguous(),
               ovvv=go[:, v, v, v].contiguous())
    del go
    Cv = C[:, nocc:]
    vvvv = torch.empty((nvir,) * 4, dtype=C.dtype, device=C.device)
    for a0 in range(0, nvir, bs):
        a1 = min(nvir, a0 + bs)
        vvvv[a0:a1] = lowmem.transform_rows(eri, Cv[:, a0:a1], Cv, Cv, Cv)
    out["vvvv"] = vvvv
    return out


def _E(mode):
    def E(spec, a, b, out=None, alpha=1.0, beta=0.0):
        return contract(spec, a, b, out=out, alpha=alpha, beta=beta, mode=mode)
    return E


def update_amps_gpu(t1, t2, eris, mode="tf32x3", level_shift=0.0):
    """One Jacobi step of the RCCSD amplitude equations; returns (t1new, t2new)."""
    E = _E(mode)
    nocc, nvir = t1.shape
    fock = eris.fock
    foo, fov, fvv = fock[:nocc, :nocc], fock[:nocc, nocc:], fock[nocc:, nocc:]
    eo, ev = eris.mo_energy[:nocc], eris.mo_energy[nocc:] + level_shift
    ovov, ovvv, ovoo, ovvo, oovv, oooo = eris.ovov, eris.ovvv, eris.ovoo, eris.ovvo, eris.oovv, eris.oooo
    t1t1 = torch.einsum("ic,jd->ijcd", t1, t1)
    tau = t2 + t1t1
    Lovov = [(2.0, ovov), (-1.0, ovov.permute(0, 3, 2, 1))]
    Xovvv = [(2.0, ovvv), (-1.0, ovvv.permute(0, 3, 2, 1))]          # [k,d,a,c]: 2(kd|ac) - (kc|ad)
    Yovoo = [(2.0, ovoo), (-1.0, ovoo.permute(2, 1, 0, 3))]          # [l,c,k,i]: 2(lc|ki) - (kc|li)
    Foo = foo + E("kcld,ilcd->ki", Lovov, tau)
    Fvv = fvv - E("kcld,klad->ac", Lovov, tau)
    Fov = fov + E("kcld,ld->kc", Lovov, t1)
    yt1 = E("lcki,lc->ki", Yovoo, t1)
    xt1 = E("kdac,kd->ac", Xovvv, t1)
    Loo = Foo + fov @ t1.T + yt1
    Lvv = Fvv - t1.T @ fov + xt1
    Foo = Foo - torch.diag(eo)
    Fvv = Fvv - torch.diag(ev)
    Loo = Loo - torch.diag(eo)
    Lvv = Lvv - torch.diag(ev)
    # T1
    t1n = (fov - 2 * t1 @ fov.T @ t1 + t1 @ Fvv.T - Foo.T @ t1 + t1 @ Fov.T @ t1 + t1 @ xt1.T - yt1.T @ t1)
    E("kc,kica->ia", Fov, [(2.0, t2), (-1.0, t2.permute(1, 0, 2, 3))], out=t1n, beta=1.0)
    E("kcai,kc->ia", ovvo, t1, out=t1n, alpha=2.0, beta=1.0)
    E("kiac,kc->ia", oovv, t1, out=t1n, alpha=-1.0, beta=1.0)
    E("kdac,ikcd->ia", Xovvv, t2, out=t1n, beta=1.0)
    E("lcki,klac->ia", Yovoo, t2, out=t1n, alpha=-1.0, beta=1.0)
    # T2
    # (ovvv^T - oovv t1) t1 without the o v^3 intermediate: the second
    # product goes through X[k,i,b,j] = sum_c oovv[k,i,b,c] t1[j,c] (o^3 v)
    tmp = E("iacb,jc->ijab", ovvv, t1)
    xk = E("kibc,jc->kibj", oovv, t1)
    E("kibj,ka->ijab", xk, t1, out=tmp, alpha=-1.0, beta=1.0)
    t2n = tmp + tmp.permute(1, 0, 3, 2)
    tmp2 = E("kcai,jc->akij", ovvo, t1)
    tmp2 += ovoo.permute(1, 3, 0, 2)
    tmp = E("akij,kb->ijab", tmp2, t1)
    t2n -= tmp + tmp.permute(1, 0, 3, 2)
    t2n += ovov.permute(0, 2, 1, 3)
    Woooo = E("lcki,jc->klij", ovoo, t1)
    E("kclj,ic->klij", ovoo, t1, out=Woooo, beta=1.0)
    E("kcld,ijcd->klij", ovov, tau, out=Woooo, beta=1.0)
    Woooo += oooo.permute(0, 2, 1, 3)
    E("klij,klab->ijab", Woooo, tau, out=t2n, beta=1.0)
    # Wvvvv . tau without forming Wvvvv
    E("acbd,ijcd->ijab", eris.vvvv, tau, out=t2n, beta=1.0)
    Zt = E("kdac,ijcd->ijka", ovvv, tau)
    tmp = E("ijka,kb->ijab", Zt, t1)
    t2n -= tmp + tmp.permute(1, 0, 3, 2)
    t1t1b = torch.einsum("id,la->ilda", t1, t1)
    half_t2_t1t1 = [(0.5, t2), (1.0, t1t1b)]
    Wvoov = ovvo.permute(2, 0, 3, 1).contiguous()
    E("kcad,id->akic", ovvv, t1, out=Wvoov, beta=1.0)
    E("kcli,la->akic", ovoo, t1, out=Wvoov, alpha=-1.0, beta=1.0)
    E("ldkc,ilda->akic", ovov, half_t2_t1t1, out=Wvoov, alpha=-1.0, beta=1.0)
    E("ldkc,ilad->akic", [(1.0, ovov), (-0.5, ovov.permute(0, 3, 2, 1))], t2, out=Wvoov, beta=1.0)
    Wvovo = oovv.permute(2, 0, 3, 1).contiguous()
    E("kdac,id->akci", ovvv, t1, out=Wvovo, beta=1.0)
    E("lcki,la->akci", ovoo, t1, out=Wvovo, alpha=-1.0, beta=1.0)
    E("lckd,ilda->akci", ovov, half_t2_t1t1, out=Wvovo, alpha=-1.0, beta=1.0)
    tmp = E("ac,ijcb->ijab", Lvv, t2)
    t2n += tmp + tmp.permute(1, 0, 3, 2)
    tmp = E("ki,kjab->ijab", Loo, t2)
    t2n -= tmp + tmp.permute(1, 0, 3, 2)
    tmp = E("akic,kjcb->ijab", [(2.0, Wvoov), (-1.0, Wvovo.permute(0, 1, 3, 2))], t2)
    t2n += tmp + tmp.permute(1, 0, 3, 2)
    tmp = E("akic,kjbc->ijab", Wvoov, t2)
    t2n -= tmp + tmp.permute(1, 0, 3, 2)
    tmp = E("bkci,kjac->ijab", Wvovo, t2)
    t2n -= tmp + tmp.permute(1, 0, 3, 2)
    eia = eo[:, None] - ev[None, :]
    return t1n / eia, t2n / (eia[:, None, :, None] + eia[None, :, None, :])


def energy_gpu(t1, t2, eris):
    nocc = t1.shape[0]
    tau = t2 + torch.einsum("ia,jb->ijab", t1, t1)
    ov = eris.ovov
    return float(2 * (eris.fock[:nocc, nocc:] * t1).sum() + 2 * torch.einsum("ijab,iajb->", tau, ov)
                 - torch.einsum("ijab,ibja->", tau, ov))


class CCSD:
    """PySCF-like closed-shell CCSD on the GPU.

    ``frozen``: number of lowest (core) orbitals kept out of the correlation
    treatment, as PySCF's integer ``frozen`` (ref: the reference's frozen-core
    branches, ccsd_gpu/gpu_ccsd_grad.py:373-374,510-518)."""

    def __init__(self, mf, precision="tf32x3", frozen=0):
        _native.require_cuda()
        self._scf = mf
        self.mol = mf.mol
        self.mo_coeff = mf.mo_coeff
        self.mo_occ = mf.mo_occ
        self.mo_energy = mf.mo_energy
        self.precision = precision
        self.max_cycle = 100
        self.conv_tol = 1e-9
        self.conv_tol_normt = 1e-7
        self.t_polish = True
        self.lambda_polish = True
        self.diis_space = 8
        self.level_shift = 0.0
        # replay the T / Lambda update bodies as CUDA graphs.  Off by default:
        # one capture per solve (eager + warm-up + capture) costs about as much
        # as it saves over the 12-20 iterations of one gradient (measured on
        # H2O and (H2O)6, cc-pVDZ)
        self.use_graphs = False
        # FP64 iteration bodies are captured once per (shape, level shift) and
        # replayed by every later solve of the same shape (integrals copied in)
        self.use_graph_cache = True
        self.verbose = 0
        self.t1 = self.t2 = self.l1 = self.l2 = None
        self.converged = self.converged_lambda = False
        self._eris = None
        self.frozen = int(frozen or 0)
        if not 0 <= self.frozen < int((np.asarray(self.mo_occ) > 0).sum()):
            raise ValueError("frozen must leave at least one active occupied orbital")

    @property
    def nocc(self):
        """Active occupied orbitals."""
        return int((np.asarray(self.mo_occ) > 0).sum()) - self.frozen

    def ao2mo(self, mo_coeff=None):
        if self._eris is None or mo_coeff is not None:
            self._eris = ao2mo_gpu(self._scf, mo_coeff, self.frozen)
        return self._eris

    def kernel(self, t1=None, t2=None, eris=None):
        eris = self.ao2mo() if eris is None else DeviceEris.wrap(eris)
        lowmem.tidy(self.mol.nao_nr())
        nocc = self.nocc
        eo, ev = eris.mo_energy[:nocc], eris.mo_energy[nocc:]
        eia = eo[:, None] - ev[None, :]
        d2 = eia[:, None, :, None] + eia[None, :, None, :]
        t1 = eris.fock[:nocc, nocc:] / eia if t1 is None else torch.as_tensor(t1, device=eia.device)
        t2 = eris.ovov.permute(0, 2, 1, 3) / d2 if t2 is None else torch.as_tensor(t2, device=eia.device)
        adiis = DIIS(self.diis_space)
        e_old = energy_gpu(t1, t2, eris)
        nov = t1.numel()
        self.converged = False
        # split precision down to its ~1e-6 noise floor, then FP64 iterations
        # (mixed-precision iterative refinement; ``t_polish = False`` skips them)
        mode = effective_mode(self.precision, nocc, t1.shape[1])
        tol_n = self.conv_tol_normt if mode == "fp64" else max(self.conv_tol_normt, 1e-6)
        self._t_history = []
        step = self._step(eris, mode)
        for it in range(self.max_cycle):
            t1n, t2n = step(t1, t2)
            normt = float(torch.sqrt(amplitude_norm_sq(t1n - t1, t2n - t2)))
            self._t_history.append((mode, normt))
            x = adiis.update(torch.cat([t1n.reshape(-1), t2n.reshape(-1)]),
                             torch.cat([(t1n - t1).reshape(-1), (t2n - t2).reshape(-1)]))
            t1, t2 = x[:nov].reshape(t1.shape), x[nov:].reshape(t2.shape)
            e = energy_gpu(t1, t2, eris)
            if normt < tol_n and abs(e - e_old) < self.conv_tol:
                if mode != "fp64" and self.t_polish and self.conv_tol_normt < tol_n:
                    mode, tol_n = "fp64", self.conv_tol_normt
                    step = self._step(eris, mode)
                    adiis = DIIS(self.diis_space)
                    e_old = e
                    continue
                # converged only if the requested tolerance was met: a split-precision
                # solve stopped at its noise floor without the FP64 polish is not
                self.converged = normt < self.conv_tol_normt
                break
            e_old = e
        check_status()
        self.normt = self._t_history[-1][1] if self._t_history else None
        self.e_corr = e
        self.t1, self.t2 = host_copy(t1), host_copy(t2)
        remember_device(self, "t1", self.t1, t1)
        remember_device(self, "t2", self.t2, t2)
        return self.e_corr, self.t1, self.t2

    def _step(self, eris, mode):
        ls = self.level_shift
        nocc = eris.ovoo.shape[0]
        nvir = eris.fock.shape[0] - nocc
        if self.use_graph_cache and not self.use_graphs and graph_cache_ok(mode, nocc, nvir):
            consts = {k: getattr(eris, k) for k in _T_CONSTS}
            key = ("T", nocc, nvir, float(ls), mode)
            return solve_step(key, lambda c, a, b: update_amps_gpu(a, b, SimpleNamespace(**c), mode, ls), consts)
        return StepGraph(lambda a, b: update_amps_gpu(a, b, eris, mode, ls), enabled=self.use_graphs)

    @property
    def e_tot(self):
        return self._scf.e_tot + self.e_corr

    def solve_lambda(self, t1=None, t2=None, l1=None, l2=None, eris=None):
        lowmem.tidy(self.mol.nao_nr())
        return solve_lambda_gpu(self, t1, t2, l1, l2, eris=self.ao2mo() if eris is None else eris,
                                mode=self.precision)

    def nuc_grad_method(self):
        from .gpu_ccsd_grad import Gradients
        return Gradients(self)
