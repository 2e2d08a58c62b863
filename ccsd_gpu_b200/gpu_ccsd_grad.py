"""CCSD analytic nuclear gradient on the GPU.

Drop-in for ``ccsd_gpu.gpu_ccsd_grad`` (ref: ccsd_gpu/gpu_ccsd_grad.py):
``_gamma1_intermediates_gpu`` (:101-126), ``_gamma2_intermediates_gpu``
(:129-246), ``_rdm2_mo2ao_gpu`` (:254-336), ``grad_elec_gpu`` (:344-586) and
``compute_ml_ccsd_forces_gpu`` (:711-739) keep their signatures and return
numpy arrays like the reference.  Everything runs on the device:

  * RDM intermediates through the contraction engine in the CC object's
    precision; MO->AO transform, all gradient contractions, the CPHF
    (Z-vector) solve and the one-electron terms in FP64;
  * the two-electron gradient term: the 2-RDM and the P x relaxed-density
    products (the reference's de_k and vhf1 terms) form one density that is
    contracted with int2e_ip1 inside the ERI kernel, shell quartet by shell
    quartet (:func:`ccsd_gpu_b200.cuda.ip1_contract.contract_int2e_ip1`); no
    derivative integral is stored (the reference stores each atom block and
    falls back to CPU libcint below nao = 50).  Imat comes from the SCF's
    resident ERIs, one-electron derivative integrals from the ``int1e``
    kernel (the reference uses CPU libcint through PySCF);
  * the Z-vector equations (e_a - e_i) x + A x = -Xvo are solved directly in
    FP64 (the reference iterates PySCF's cphf.solve to 1e-9).
``CCSDEnergy`` wraps E(R) in a torch.autograd.Function whose backward is
this hand-written adjoint (Lambda + RDM + int2e_ip1 . Gamma + Z-vector).
"""
import numpy as np
import torch

from . import _native, lowmem
from .contract import check_status, clear_pack_cache, contract
from .gpu_ccsd_lambda import device_amp
from .cuda.ip1_contract import contract_int2e_ip1, contract_int2e_ip1_rows
from .int1e import intor1e


def _t(x, dev):
    if isinstance(x, torch.Tensor):
        return x.to(dev, dtype=torch.float64)
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=dev)


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def _E(mode):
    def E(spec, a, b, out=None, alpha=1.0, beta=0.0):
        return contract(spec, a, b, out=out, alpha=alpha, beta=beta, mode=mode)
    return E


def _mode(mycc):
    return getattr(mycc, "precision", None) or "tf32x3"


def _gamma1_intermediates_gpu(mycc, t1, t2, l1, l2):
    """(doo, dov, dvo, dvv) (ref: ccsd_gpu/gpu_ccsd_grad.py:101-126)."""
    E = _E(_mode(mycc))
    dev = _dev()
    t1, t2, l1, l2 = (_t(x, dev) for x in (t1, t2, l1, l2))
    theta = [(2.0, t2), (-1.0, t2.permute(0, 1, 3, 2))]
    doo = -t1 @ l1.T
    doo = doo.T.contiguous()           # doo[i,j] = -sum_a t1[j,a] l1[i,a]
    E("jkab,ikab->ij", theta, l2, out=doo, alpha=-1.0, beta=1.0)
    dvv = t1.T @ l1
    E("jica,jicb->ab", theta, l2, out=dvv, beta=1.0)
    xtv = t1 @ l1.T
    xt1 = E("mnef,inef->mi", l2, theta)
    xt2 = E("mnaf,mnef->ea", l2, theta)
    dvo = t1.T - (xtv @ t1).T - (xt1.T @ t1).T - (t1 @ xt2.T).T
    E("imae,me->ai", theta, l1, out=dvo, beta=1.0)
    return doo, l1.clone(), dvo.contiguous(), dvv


def _gamma2_intermediates_gpu(mycc, t1, t2, l1, l2):
    """(dovov, dvvvv, doooo, doovv, dovvo, None, dovvv, dooov)
    (ref: ccsd_gpu/gpu_ccsd_grad.py:129-246)."""
    E = _E(_mode(mycc))
    dev = _dev()
    t1, t2, l1, l2 = (_t(x, dev) for x in (t1, t2, l1, l2))
    theta = [(2.0, t2), (-1.0, t2.permute(0, 1, 3, 2))]
    pvOOv = E("ikca,jkcb->aijb", l2, t2)
    pvoOV = E("ikca,jkbc->aijb", l2, t2, alpha=-1.0)
    E("ikac,jkbc->aijb", l2, theta, out=pvoOV, beta=1.0)
    moo = 2 * torch.einsum("dljd->jl", pvOOv) + torch.einsum("dljd->jl", pvoOV)
    mvv = 2 * torch.einsum("blld->db", pvOOv) + torch.einsum("blld->db", pvoOV)
    mia = E("kc,ikac->ia", l1, theta)
    mab = l1.T @ t1
    mij = t1 @ l1.T + 0.5 * moo
    tau = t2 + torch.einsum("ia,jb->ijab", t1, t1)
    goooo = E("ijab,klab->ijkl", tau, l2, alpha=0.5)
    doooo = 2 * goooo.permute(0, 2, 1, 3) - goooo.permute(0, 3, 1, 2)
    gooov = E("kc,cija->jkia", t1, pvOOv)
    E("jc,cika->jkia", t1, pvoOV, out=gooov, alpha=-1.0, beta=1.0)
    gooov -= 0.5 * torch.einsum("ji,ka->jkia", moo, t1)
    E("la,jkil->jkia", t1, goooo, out=gooov, alpha=2.0, beta=1.0)
    E("ib,jkba->jkia", l1, tau, out=gooov, alpha=-1.0, beta=1.0)
    E("jkba,ib->jkia", l2, t1, out=gooov, alpha=-1.0, beta=1.0)
    dooov = 2 * gooov.permute(0, 2, 1, 3) - gooov.permute(1, 2, 0, 3)
    goovv = torch.einsum("ia,jb->ijab", mia, t1) + 0.5 * tau + 0.5 * l2
    E("ijkl,klab->ijab", goooo, tau, out=goovv, beta=1.0)
    E("jk,ikab->ijab", mij, tau, out=goovv, alpha=-1.0, beta=1.0)
    E("cb,ijac->ijab", mab, t2, out=goovv, alpha=-1.0, beta=1.0)
    E("bd,ijad->ijab", mvv, tau, out=goovv, alpha=-0.5, beta=1.0)
    t1t1 = torch.einsum("jc,kb->jkcb", t1, t1)
    gOvvO = pvOOv.permute(1, 0, 3, 2).contiguous()
    E("kiac,jkcb->iabj", l2, t1t1, out=gOvvO, beta=1.0)
    govVO = torch.einsum("ia,jb->iabj", l1, t1) + pvoOV.permute(1, 0, 3, 2)
    E("ikac,jkcb->iabj", l2, t1t1, out=govVO, alpha=-1.0, beta=1.0)
    dovvo = 2 * govVO + gOvvO
    doovv = (-2 * gOvvO - govVO).permute(3, 0, 1, 2).contiguous()
    tau_h = tau - 0.5 * t2
    E("dlib,jlda->ijab", pvOOv, tau_h, out=goovv, beta=1.0)
    E("dlia,jldb->ijab", pvoOV, tau_h, out=goovv, alpha=-1.0, beta=1.0)
    E("dlia,jlbd->ijab", [(1.0, pvoOV), (0.5, pvOOv)], t2, out=goovv, beta=1.0)
    dovov = 2 * goovv.permute(0, 2, 1, 3) - goovv.permute(1, 2, 0, 3)
    gvvvv = E("ijab,ijcd->abcd", l2, tau)          # l2 . (t2 + t1 t1)
    dvvvv = torch.empty_like(gvvvv)                 # one nvir^4 temporary at most
    dvvvv.copy_(gvvvv.permute(0, 2, 1, 3))
    dvvvv.sub_(gvvvv.permute(0, 3, 1, 2), alpha=0.5)
    del gvvvv
    # gvovv[a,i,b,c] = -sum_d gvvvv[a,d,b,c] t1[i,d], evaluated as
    # -sum_kl (sum_d l2[k,l,a,d] t1[i,d]) tau[k,l,b,c]: one tensor-core GEMM
    # instead of a skinny product that re-reads a permuted nvir^4 array
    xl2t1 = E("klad,id->klai", l2, t1)
    gvovv = E("klai,klbc->aibc", xl2t1, tau, alpha=-1.0)
    E("akic,kb->aibc", pvoOV, t1, out=gvovv, beta=1.0)
    E("akib,kc->aibc", pvOOv, t1, out=gvovv, alpha=-1.0, beta=1.0)
    E("ja,jibc->aibc", l1, tau, out=gvovv, beta=1.0)
    gvovv += 0.5 * torch.einsum("ba,ic->aibc", mvv, t1)
    E("ja,jibc->aibc", t1, l2, out=gvovv, beta=1.0)
    dovvv = 2 * gvovv.permute(1, 3, 0, 2) - gvovv.permute(1, 2, 0, 3)
    return (dovov.contiguous(), dvvvv.contiguous(), doooo.contiguous(), doovv, dovvo.contiguous(), None,
            dovvv.contiguous(), dooov.contiguous())


def _rdm2_mo(d2):
    """Full MO 2-RDM in the reference's layout (ref: ccsd_gpu/gpu_ccsd_grad.py:272-311)."""
    return _rdm2_mo_raw(d2).permute(1, 0, 3, 2)


def _rdm2_mo_raw(d2):
    """The MO 2-RDM before the final (1, 0, 3, 2) index permutation, contiguous.
    The symmetrised AO 2-RDM (``_rdm2_ao``) is the same from either, since its
    symmetrisation over (p <-> q) and (r <-> s) absorbs that permutation."""
    dovov, dvvvv, doooo, doovv, dovvo, _, dovvv, dooov = d2
    nocc, nvir = dovov.shape[:2]
    n = nocc + nvir
    o, v = slice(0, nocc), slice(nocc, n)
    dm2 = torch.zeros((n,) * 4, dtype=torch.float64, device=dovov.device)
    dm2[o, v, o, v] = dovov + dovov.permute(2, 3, 0, 1)
    dm2[v, o, v, o] = dm2[o, v, o, v].permute(1, 0, 3, 2)
    dm2[o, o, v, v] = doovv + doovv.permute(1, 0, 3, 2)
    dm2[v, v, o, o] = dm2[o, o, v, v].permute(2, 3, 0, 1)
    dm2[o, v, v, o] = dovvo + dovvo.permute(3, 2, 1, 0)
    dm2[v, o, o, v] = dm2[o, v, v, o].permute(1, 0, 3, 2)
    # the nvir^4 block in place (no nvir^4 temporaries)
    vvvv = dm2[v, v, v, v]
    vvvv.copy_(dvvvv)
    vvvv.add_(dvvvv.permute(1, 0, 3, 2))
    vvvv.mul_(2.0)
    dm2[o, o, o, o] = 2 * (doooo + doooo.permute(1, 0, 3, 2))
    dm2[o, v, v, v] = dovvv
    dm2[v, v, o, v] = dovvv.permute(2, 3, 0, 1)
    dm2[v, v, v, o] = dovvv.permute(3, 2, 1, 0)
    dm2[v, o, v, v] = dovvv.permute(1, 0, 3, 2)
    dm2[o, o, o, v] = dooov
    dm2[o, v, o, o] = dooov.permute(2, 3, 0, 1)
    dm2[o, o, v, o] = dooov.permute(1, 0, 3, 2)
    dm2[v, o, o, o] = dooov.permute(3, 2, 1, 0)
    return dm2


def _rdm2_ao_rows(M, CaT, p0, p1):
    """Rows [p0, p1) of the symmetrised AO 2-RDM (``_rdm2_ao``) from the raw MO
    2-RDM M (``_rdm2_mo_raw``) and CaT = C_active^T, without the (nao,)*4
    tensor: rows and columns of the AO transform (lowmem.transform_rows and
    transform_cols1), then the (p <-> q, r <-> s) symmetrisation of the rows."""
    g = lowmem.transform_rows(M, CaT[:, p0:p1], CaT, CaT, CaT)
    g += lowmem.transform_cols1(M, CaT, CaT[:, p0:p1], CaT, CaT)
    return 0.5 * (g + g.transpose(2, 3))


def _add_hf_terms(gam, P, dm1p, r0=0):
    """gam (rows [r0, r0 + len(gam)) of an (n,)*4 density) += the HF-like
    products of P and the relaxed density dm1p, symmetrised in k <-> l
    (ref: ccsd_gpu/gpu_ccsd_grad.py:416-500, de_k and vhf1): broadcast
    in-place updates, no (n,)*4 temporaries."""
    Pr, Dr = P[r0:r0 + gam.shape[0]], dm1p[r0:r0 + gam.shape[0]]
    gam.addcmul_(Pr[:, :, None, None], dm1p[None, None])                        # P_ij D_kl
    gam.addcmul_(Dr[:, :, None, None], P[None, None])                           # D_ij P_kl
    gam.addcmul_(Pr[:, None, None, :], dm1p.T[None, :, :, None], value=-0.25)   # P_il D_kj
    gam.addcmul_(Pr[:, None, :, None], dm1p.T[None, :, None, :], value=-0.25)   # P_ik D_lj
    gam.addcmul_(Dr[:, None, None, :], P[None, :, :, None], value=-0.25)        # D_il P_jk
    gam.addcmul_(Dr[:, None, :, None], P[None, :, None, :], value=-0.25)        # D_ik P_jl


def _rdm2_ao(d2, mo_coeff):
    """Symmetrised AO 2-RDM, full (nao,)*4, FP64."""
    C = mo_coeff
    g = _rdm2_mo(d2)
    g = torch.einsum("pi,ijkl->pjkl", C, g)
    g = torch.einsum("qj,pjkl->pqkl", C, g)
    g = torch.einsum("rk,pqkl->pqrl", C, g)
    g = torch.einsum("sl,pqrl->pqrs", C, g)
    g = g + g.permute(1, 0, 2, 3)
    return 0.5 * (g + g.permute(0, 1, 3, 2))


def _rdm2_mo2ao_gpu(mycc, d2, mo_coeff):
    """Lower-triangle packed AO 2-RDM (nao_pair, nao_pair) (ref: ccsd_gpu/gpu_ccsd_grad.py:254-336)."""
    C = _t(mo_coeff, _dev())
    dm2 = _rdm2_ao(d2, C)
    nao = C.shape[0]
    r, c = torch.tril_indices(nao, nao, device=C.device)
    p = r * nao + c
    return dm2.reshape(nao * nao, nao * nao)[p[:, None], p[None, :]]


def grad_elec_gpu(mycc, t1, t2, l1, l2, atmlst=None, verbose=None):
    """Electronic part of the CCSD gradient, numpy (natm, 3)
    (ref: ccsd_gpu/gpu_ccsd_grad.py:344-586)."""
    _native.require_cuda()
    dev = _dev()
    mf = mycc._scf
    mol = mycc.mol
    C = _t(mf.mo_coeff, dev)
    e = _t(mf.mo_energy, dev)
    nao, nmo = C.shape
    nocc = int((np.asarray(mf.mo_occ) > 0).sum())
    # frozen core: the amplitudes span occupied orbitals nf..nocc-1 (ref:
    # ccsd_gpu/gpu_ccsd_grad.py:373-374); no frozen virtuals
    nf = nocc - int(np.shape(t1)[0])
    if nf < 0 or int(np.shape(t1)[1]) != nmo - nocc:
        raise ValueError("amplitudes do not match the SCF orbitals (only frozen core orbitals are supported)")
    Co, Cv = C[:, :nocc], C[:, nocc:]
    # large molecules (four more (nao,)*4 tensors would not fit): the AO
    # 2-RDM is never formed whole; it is built atom block by atom block, once
    # for Imat and once for the ip1 contraction (the reference streams its
    # gradient by shell blocks, ref: ccsd_gpu/gpu_ccsd_grad.py:416-432)
    lean = lowmem.lean(4, nao, dev)
    if lean:
        clear_pack_cache()
        if getattr(mycc, "_eris", None) is not None:
            mycc._eris = None           # rebuilt by mycc.ao2mo() on demand
        torch.cuda.empty_cache()
    eri = mf.eri                        # (recomputed here if the ao2mo released it)
    doo, dov, dvo, dvv = _gamma1_intermediates_gpu(mycc, t1, t2, l1, l2)
    d2 = _gamma2_intermediates_gpu(mycc, t1, t2, l1, l2)
    P = 2 * Co @ Co.T
    atmlst = range(mol.natm) if atmlst is None else atmlst
    off = mol.offset_nr_by_atom()
    de = torch.zeros((mol.natm, 3), dtype=torch.float64, device=dev)
    if lean:
        M = _rdm2_mo_raw(d2)
        del d2
        CaT = C[:, nf:].T.contiguous()
        Imat = torch.zeros((nao, nao), dtype=torch.float64, device=dev)
        for a in range(mol.natm):
            p0, p1 = int(off[a][2]), int(off[a][3])
            if p1 > p0:
                rows = _rdm2_ao_rows(M, CaT, p0, p1)
                Imat += 0.5 * torch.einsum("ipkl,iqkl->pq", eri[p0:p1], rows)
                del rows
    else:
        dm2 = _rdm2_ao(d2, C[:, nf:])
        del d2
        Imat = 0.5 * torch.einsum("ipkl,iqkl->pq", eri, dm2)
    S = mf.get_ovlp()
    Imat = -(C.T @ Imat @ S @ C)
    dm1mo = torch.zeros((nmo, nmo), dtype=torch.float64, device=dev)
    dm1mo[nf:nocc, nf:nocc] = doo + doo.T
    dm1mo[nocc:, nocc:] = dvv + dvv.T
    if nf:
        # frozen-active occupied block of the relaxed density
        # (ref: ccsd_gpu/gpu_ccsd_grad.py:510-518)
        dco = Imat[:nf, nf:nocc] / (e[:nf, None] - e[None, nf:nocc])
        dm1mo[:nf, nf:nocc] = dco
        dm1mo[nf:nocc, :nf] = dco.T
    dm1 = C @ dm1mo @ C.T
    vhf = mf.get_veff(dm=dm1) * 2
    Xvo = Cv.T @ vhf @ Co + Imat[:nocc, nocc:].T - Imat[nocc:, :nocc]
    dvo_z = _zvector(mf, e, Co, Cv, Xvo)
    dm1mo[nocc:, :nocc] += dvo_z
    dm1mo[:nocc, nocc:] += dvo_z.T
    Imat[nocc:, :nocc] = Imat[:nocc, nocc:].T
    im1 = C @ Imat @ C.T
    s1 = -intor1e(mol, "int1e_ipovlp")
    h1 = -(intor1e(mol, "int1e_ipkin") + intor1e(mol, "int1e_ipnuc"))
    zeta = 0.5 * (e[:, None] + e[None, :])
    zeta[nocc:, :nocc] = e[:nocc]
    zeta[:nocc, nocc:] = e[:nocc].reshape(-1, 1)
    zeta = C @ (zeta * dm1mo) @ C.T
    dm1 = C @ dm1mo @ C.T
    p1 = Co @ Co.T
    vhf_s1occ = p1 @ mf.get_veff(dm=dm1 + dm1.T) @ p1
    dm1p = P + 2 * dm1
    dm1 = dm1 + P
    zeta = zeta + (Co * (2 * e[:nocc])) @ Co.T
    # Two-electron term: the 2-RDM and the HF-like products of P with the
    # relaxed density (ref: ccsd_gpu/gpu_ccsd_grad.py:416-500, de_k and vhf1)
    # in one density, symmetrised in k <-> l, contracted with int2e_ip1 that
    # is recomputed shell quartet by shell quartet and never stored.
    # dm2 is already symmetric in k <-> l and so are P (x) dm1p and dm1p (x) P
    # (both densities are symmetric); the exchange products are symmetrised
    # term by term.  Broadcast in-place updates: no (nao,)*4 temporaries.
    if lean:
        for a in range(mol.natm):
            p0, p1 = int(off[a][2]), int(off[a][3])
            if p1 > p0:
                rows = _rdm2_ao_rows(M, CaT, p0, p1)
                _add_hf_terms(rows, P, dm1p, p0)
                de[a] -= contract_int2e_ip1_rows(mol, rows, a)
                del rows
        del M
    else:
        gam = dm2
        del dm2
        _add_hf_terms(gam, P, dm1p)
        de -= contract_int2e_ip1(mol, gam)
        del gam
    charges = mol.atom_charges()
    for a in atmlst:
        _, _, p0, p1_ = (int(v) for v in off[a])
        vr = -float(charges[a]) * intor1e(mol, "int1e_iprinv", origin_atom=a)
        vr[:, p0:p1_] += h1[:, p0:p1_]
        h1ao = vr + vr.transpose(1, 2)
        s1a = s1[:, p0:p1_]
        de[a] += torch.einsum("xij,ij->x", s1a, im1[p0:p1_])
        de[a] += torch.einsum("xji,ij->x", s1a, im1[:, p0:p1_])
        de[a] += torch.einsum("xij,ji->x", h1ao, dm1)
        de[a] -= torch.einsum("xij,ij->x", s1a, zeta[p0:p1_])
        de[a] -= torch.einsum("xji,ij->x", s1a, zeta[:, p0:p1_])
        de[a] -= 2 * torch.einsum("xij,ij->x", s1a, vhf_s1occ[p0:p1_])
    # the RDM and gvovv contractions ran on the tensor cores: an expired
    # pipeline wait leaves their tiles unwritten, so raise instead of
    # returning a gradient built from them
    check_status(dev)
    return de[list(atmlst)].cpu().numpy()


def _zvector(mf, e, Co, Cv, Xvo):
    """Solve (e_a - e_i) x_ai + [2 Cv^T veff(Cv x Co^T + h.c.) Co]_ai = -Xvo_ai in FP64.

    Small systems: the orbital Hessian is built column-block by column-block
    and solved directly; larger ones use conjugate gradients (the operator is
    symmetric positive definite for a stable closed-shell HF reference)."""
    nocc, nvir = Co.shape[1], Cv.shape[1]
    eia = (e[nocc:, None] - e[None, :nocc])

    def apply(X):
        dm = Cv @ X @ Co.T
        return eia * X + 2 * (Cv.T @ mf.get_veff(dm=dm + dm.T) @ Co)

    b = -Xvo
    x = b / eia
    r = b - apply(x)
    z = r / eia
    p = z.clone()
    rz = (r * z).sum()
    bn = float(b.norm())
    for _ in range(200):
        Ap = apply(p)
        alpha = rz / (p * Ap).sum()
        x = x + alpha * p
        r = r - alpha * Ap
        if float(r.norm()) < 1e-12 * max(bn, 1.0):
            break
        z = r / eia
        rz_new = (r * z).sum()
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x


class Gradients:
    """``mycc.nuc_grad_method()``: electronic + nuclear gradient (natm, 3)."""

    def __init__(self, mycc):
        self.base = mycc

    def kernel(self, t1=None, t2=None, l1=None, l2=None):
        cc = self.base
        t1 = cc.t1 if t1 is None else t1
        t2 = cc.t2 if t2 is None else t2
        if l1 is None or l2 is None:
            if cc.l1 is None:
                cc.solve_lambda()
            l1, l2 = cc.l1, cc.l2
        t1, t2 = device_amp(cc, "t1", t1), device_amp(cc, "t2", t2)
        l1, l2 = device_amp(cc, "l1", l1), device_amp(cc, "l2", l2)
        self.de = grad_elec_gpu(cc, t1, t2, l1, l2) + cc.mol.grad_nuc()
        return self.de


def compute_ml_ccsd_forces_gpu(mf, t1, t2, l1, l2, precision="tf32x3"):
    """dE/dR (natm, 3) in Eh/bohr, electronic + nuclear (ref: ccsd_gpu/gpu_ccsd_grad.py:711-739).

    As in the reference this is the gradient (not its negative)."""
    from .ccsd import CCSD
    nf = int((np.asarray(mf.mo_occ) > 0).sum()) - int(np.shape(t1)[0])     # frozen core from the shapes
    mycc = CCSD(mf, precision=precision, frozen=nf)
    mycc.t1, mycc.t2, mycc.l1, mycc.l2 = t1, t2, l1, l2
    mycc.converged = mycc.converged_lambda = True
    de = grad_elec_gpu(mycc, t1, t2, l1, l2)
    check_status()
    return np.array(de + mf.nuc_grad_method().grad_nuc())


class CCSDEnergy(torch.autograd.Function):
    """E_CCSD(R) as a differentiable function of the nuclear coordinates (bohr).

    forward: RHF + CCSD at the given geometry (GPU).  backward: the adjoint --
    Lambda solve, RDMs, int2e_ip1 . Gamma, Z-vector and one-electron terms
    (:func:`grad_elec_gpu`) plus the nuclear term.  Usage::

        e = CCSDEnergy.apply(coords, mol_template, "tf32x3")
        e.backward()            # coords.grad = dE/dR
    """

    @staticmethod
    def forward(ctx, coords, mol, precision="tf32x3", frozen=0, polish=True):
        from .ccsd import CCSD
        from .scf import RHF
        m = mol.copy().set_geom_(coords.detach().cpu().numpy())
        mf = RHF(m).run()
        cc = CCSD(mf, precision=precision, frozen=frozen)
        cc.t_polish = cc.lambda_polish = bool(polish)
        cc.kernel()
        ctx.cc = cc
        return torch.tensor(cc.e_tot, dtype=torch.float64, device=coords.device)

    @staticmethod
    def backward(ctx, gout):
        g = ctx.cc.nuc_grad_method().kernel()
        return gout * torch.as_tensor(g, dtype=torch.float64, device=gout.device), None, None, None, None
