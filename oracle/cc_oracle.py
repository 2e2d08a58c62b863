"""ORACLE -- test infrastructure only.

numpy restatement (unblocked, full tensors) of the reference's CCSD Lambda and
density-matrix path:
  * make_intermediates  ref: ccsd_gpu/gpu_ccsd_lambda.py:68-209
  * update_lambda       ref: ccsd_gpu/gpu_ccsd_lambda.py:212-337 (vvvv ladder
    sum_cd l2[ijcd] (ac|bd) included, as PySCF's _add_vvvv computes it)
  * gamma1              ref: ccsd_gpu/gpu_ccsd_grad.py:101-126
  * gamma2              ref: ccsd_gpu/gpu_ccsd_grad.py:129-246
  * rdm2_mo2ao          ref: ccsd_gpu/gpu_ccsd_grad.py:254-336
The reference evaluates the same closed-shell RCCSD Lambda equations as PySCF's
ccsd_lambda / ccsd_rdm (spin-adapted, chemist-notation integrals); the index
equations below are those equations, written without the virtual-index
blocking and memory management.

MO integral blocks follow PySCF: ovoo[i,a,j,k] = (ia|jk), ovvo[i,a,b,j] = (ia|bj),
oovv[i,j,a,b] = (ij|ab), ovvv[i,a,b,c] = (ia|bc), oooo, vvvv likewise.
"""
from types import SimpleNamespace

import numpy as np

es = lambda s, *a: np.einsum(s, *a, optimize=True)   # noqa: E731


def mo_blocks(g, nocc):
    """Chemist-notation MO integral blocks from a full (nmo,)*4 tensor."""
    o, v = slice(0, nocc), slice(nocc, g.shape[0])
    return SimpleNamespace(oooo=g[o, o, o, o], ovoo=g[o, v, o, o], ovvo=g[o, v, v, o], oovv=g[o, o, v, v],
                           ovov=g[o, v, o, v], ovvv=g[o, v, v, v], vvvv=g[v, v, v, v])


def make_intermediates(t1, t2, fock, eris):
    nocc, nvir = t1.shape
    foo, fov, fvv = fock[:nocc, :nocc], fock[:nocc, nocc:], fock[nocc:, nocc:]
    ovvv, ovoo, ovvo, oovv, oooo = eris.ovvv, eris.ovoo, eris.ovvo, eris.oovv, eris.oooo
    vvov = ovvv.transpose(2, 3, 0, 1)
    voov = ovvo.transpose(1, 0, 3, 2)
    tau = t2 + es("ia,jb->ijab", t1, t1)
    # one-particle intermediates
    w1 = fvv - es("ja,jb->ba", fov, t1)
    w2 = foo + es("ib,jb->ij", fov, t1)
    w3 = 2 * es("kc,jkbc->bj", fov, t2) + fov.T - es("kc,kjbc->bj", fov, t2) + es("kc,kb,jc->bj", fov, t1, t1)
    w4 = fov.copy()
    w1 = w1 + 2 * es("jcba,jc->ba", ovvv, t1) - es("jabc,jc->ba", ovvv, t1)
    theta_b = 2 * t2 - t2.transpose(1, 0, 2, 3)
    w3 = w3 + es("jkcd,kdcb->bj", theta_b, ovvv)
    w2 = w2 + 2 * es("kbij,kb->ij", ovoo, t1) - es("ibkj,kb->ij", ovoo, t1)
    w3 = w3 - es("lckj,klcb->bj", ovoo, 2 * t2.transpose(1, 0, 2, 3) - t2)
    g2voov = 2 * voov - voov.transpose(0, 2, 1, 3)
    x4 = es("ckld,ld->kc", g2voov, t1)
    w1 = w1 - es("ckja,kjcb->ba", g2voov, t2) - es("ja,jb->ba", x4, t1)
    w2 = w2 + es("jkbc,bikc->ij", t2, g2voov) + es("ib,jb->ij", x4, t1)
    w3 = w3 + t1.T @ x4 @ t1.T
    w4 = w4 + x4
    # two-particle intermediates
    VOov = es("bjld,klcd->bjkc", g2voov, t2) - es("bjld,kldc->bjkc", voov, t2) + voov
    vOOv = es("bljd,kldc->bjkc", voov, t2) - oovv.transpose(2, 1, 0, 3)
    wVOov = (es("jbcd,kd->bjkc", ovvv, t1) - es("jbkl,lc->bjkc", ovoo, t1)
             - es("bjld,kd,lc->bjkc", voov, t1, t1) + VOov)
    wvOOv = (-es("cbjd,kd->cjkb", vvov, t1) + es("lbjk,lc->bjkc", ovoo, t1)
             + es("bljd,kd,lc->bjkc", voov, t1, t1) + vOOv)
    ov1 = 2 * vOOv + VOov
    ov2 = 2 * VOov + vOOv
    woooo = es("lc,jcik->ijkl", t1, ovoo)
    woooo = woooo + woooo.transpose(1, 0, 3, 2) + es("cijd,klcd->ijkl", voov, tau) + oooo.transpose(0, 2, 1, 3)
    g2vovv = 2 * vvov.transpose(0, 2, 1, 3) - vvov.transpose(0, 2, 3, 1)
    g2ovoo = 2 * ovoo - ovoo.transpose(2, 1, 0, 3)
    vcjik = es("jlcb,lbki->cjki", theta_b, g2ovoo)
    wvooo = (es("cibd,jkbd->ckij", g2vovv, tau) + 2 * ovoo.transpose(1, 3, 2, 0) - ovoo.transpose(1, 0, 2, 3)
             - 1.5 * es("klbc,iblj->ckij", t2, ovoo) + vcjik.transpose(0, 3, 2, 1) - 0.5 * vcjik
             - es("jb,bikc->ckij", t1, ov1) + es("kb,bijc->ckij", t1, ov2))
    g2vvov = 2 * vvov - ovvv.transpose(1, 2, 0, 3)
    vackb = es("acjd,kjbd->ackb", g2vvov, 2 * t2 - t2.transpose(0, 1, 3, 2))
    wvvov = (-1.5 * es("jabd,jkcd->abkc", ovvv, t2) + 2 * vvov.transpose(0, 3, 2, 1) - vvov
             + vackb.transpose(0, 3, 2, 1) - 0.5 * vackb
             + es("ajkc,jb->abkc", ov1, t1) - es("ajkb,jc->abkc", ov2, t1)
             + es("laki,klbc->abic", g2ovoo, tau))
    w3 = w3 + es("ckjb,kc->bj", ov2, t1) + es("bc,jc->bj", w1, t1) - es("kj,kb->bj", w2, t1)
    return SimpleNamespace(w1=w1, w2=w2, w3=w3, w4=w4, woooo=woooo, wvooo=wvooo, wVOov=wVOov,
                           wvOOv=wvOOv, wvvov=wvvov)


def vvvv_ladder(l2, vvvv):
    """sum_cd l2[i,j,c,d] (ac|bd)."""
    return es("ijcd,acbd->ijab", l2, vvvv)


def update_lambda(t1, t2, l1, l2, fock, mo_energy, eris, imds, level_shift=0.0):
    nocc, nvir = t1.shape
    fov = fock[:nocc, nocc:]
    eo, ev = mo_energy[:nocc], mo_energy[nocc:] + level_shift
    ovvv, ovoo, ovvo, oovv = eris.ovvv, eris.ovoo, eris.ovvo, eris.oovv
    voov = ovvo.transpose(1, 0, 3, 2)
    theta = 2 * t2 - t2.transpose(0, 1, 3, 2)
    mba = es("klca,klcb->ba", l2, theta)
    mij = es("ikcd,jkcd->ij", l2, theta)
    mba1 = es("jc,jb->bc", l1, t1) + mba
    mij1 = es("kb,jb->kj", l1, t1) + mij
    mia1 = (t1 + 2 * es("kc,jkbc->jb", l1, t2) - es("kc,jkcb->jb", l1, t2) - t1 @ l1.T @ t1
            - es("bd,jd->jb", mba, t1) - es("lj,lb->jb", mij, t1))
    lad = vvvv_ladder(l2, eris.vvvv)
    l1n = 2 * es("ijab,jb->ia", lad, t1) - es("jiab,jb->ia", lad, t1)
    l2n = 0.5 * lad
    w1 = imds.w1 - np.diag(ev)
    w2 = imds.w2 - np.diag(eo)
    l1n = l1n + fov + l1 @ w1 - es("ja,ij->ia", l1, w2) - mij @ imds.w4 - es("ca,ic->ia", mba, imds.w4)
    l1n = l1n + 2 * es("ijab,bj->ia", l2, imds.w3) - es("ijba,bj->ia", l2, imds.w3)
    l2n = l2n + es("ia,jb->ijab", l1, imds.w4) + es("jibc,ca->jiba", l2, w1) - es("jk,kiba->jiba", w2, l2)
    l1n = l1n - 2 * es("iajk,kj->ia", ovoo, mij1) + es("jaik,kj->ia", ovoo, mij1)
    l2n = l2n - es("jbki,ka->jiba", ovoo, l1)
    tau = t2 + es("ia,jb->ijab", t1, t1)
    l2tau = es("ijcd,klcd->ijkl", l2, tau)
    l2t1 = es("jidc,kc->ijkd", l2, t1)
    l1n = l1n - es("jb,jiab->ia", l1, oovv)
    l1n = l1n + 2 * es("iabc,bc->ia", ovvv, mba1) - es("ibca,bc->ia", ovvv, mba1)
    l2n = l2n + es("jbac,ic->jiba", ovvv, l1)
    m4 = es("ijkd,kadb->ijab", l2t1, ovvv)
    l2n = l2n - m4
    l1n = (l1n - 2 * es("ijab,jb->ia", m4, t1) - 2 * es("ijab,ia->jb", m4, t1)
           + es("jiab,jb->ia", m4, t1) + es("jiab,ia->jb", m4, t1))
    l1n = l1n + 2 * es("jb,aijb->ia", l1, voov)
    l2n = l2n + 0.5 * voov.transpose(1, 2, 0, 3) - es("bjic,ca->jiba", voov, mba1) - es("bjka,ik->jiba", voov, mij1)
    l1n = l1n + 2 * es("aijb,jb->ia", voov, mia1) - es("bija,jb->ia", voov, mia1)
    m4 = es("ijkl,aklb->ijab", l2tau, voov)
    l2n = l2n + 0.5 * m4
    l1n = l1n + 2 * es("ijab,jb->ia", m4, t1) - es("ijba,jb->ia", m4, t1)
    l1n = l1n - es("ckij,jkca->ia", imds.wvooo, l2) + es("abkc,kibc->ia", imds.wvvov, l2)
    tmp = l2.transpose(0, 2, 1, 3) - 0.5 * l2.transpose(0, 3, 1, 2)
    l2n = l2n + es("iakc,bjkc->jiba", tmp, 2 * imds.wVOov + imds.wvOOv)
    tmp = es("jkca,bikc->jiba", l2, imds.wvOOv)
    l2n = l2n + tmp + 0.5 * tmp.transpose(1, 0, 2, 3)
    m3 = es("ijkl,klab->ijab", imds.woooo, l2)
    l2n = l2n + 0.5 * m3
    l1n = l1n + 2 * es("ijab,jb->ia", m3, t1) - es("ijba,jb->ia", m3, t1)
    eia = eo[:, None] - ev[None, :]
    l1n = l1n / eia
    l2n = (l2n + l2n.transpose(1, 0, 3, 2)) / (eia[:, None, :, None] + eia[None, :, None, :])
    return l1n, l2n


def gamma1(t1, t2, l1, l2):
    theta = 2 * t2 - t2.transpose(0, 1, 3, 2)
    doo = -es("ja,ia->ij", t1, l1) - es("jkab,ikab->ij", theta, l2)
    dvv = es("ia,ib->ab", t1, l1) + es("jica,jicb->ab", theta, l2)
    xtv = es("ie,me->im", t1, l1)
    xt1 = es("mnef,inef->mi", l2, theta)
    xt2 = es("mnaf,mnef->ea", l2, theta)
    dvo = (t1.T - es("im,ma->ai", xtv, t1) + es("imae,me->ai", theta, l1) - es("mi,ma->ai", xt1, t1)
           - es("ie,ae->ai", t1, xt2))
    return doo, l1.copy(), dvo, dvv


def gamma2(t1, t2, l1, l2):
    """(dovov, dvvvv, doooo, doovv, dovvo, dvvov=None, dovvv, dooov)."""
    theta = 2 * t2 - t2.transpose(0, 1, 3, 2)
    pvOOv = es("ikca,jkcb->aijb", l2, t2)
    pvoOV = -es("ikca,jkbc->aijb", l2, t2) + es("ikac,jkbc->aijb", l2, theta)
    moo = 2 * es("dljd->jl", pvOOv) + es("dljd->jl", pvoOV)
    mvv = 2 * es("blld->db", pvOOv) + es("blld->db", pvoOV)
    mia = 2 * es("kc,ikac->ia", l1, t2) - es("kc,ikca->ia", l1, t2)
    mab = es("kc,kb->cb", l1, t1)
    mij = es("kc,jc->jk", l1, t1) + 0.5 * moo
    tau = es("ia,jb->ijab", t1, t1) + t2
    goooo = 0.5 * es("ijab,klab->ijkl", tau, l2)
    doooo = 2 * goooo.transpose(0, 2, 1, 3) - goooo.transpose(0, 3, 1, 2)
    gooov = (es("kc,cija->jkia", t1, pvOOv) - es("jc,cika->jkia", t1, pvoOV) - 0.5 * es("ji,ka->jkia", moo, t1)
             + 2 * es("la,jkil->jkia", t1, goooo) - es("ib,jkba->jkia", l1, tau) - es("jkba,ib->jkia", l2, t1))
    dooov = 2 * gooov.transpose(0, 2, 1, 3) - gooov.transpose(1, 2, 0, 3)
    goovv = (es("ia,jb->ijab", mia, t1) + es("ijkl,klab->ijab", goooo, tau) - es("jk,ikab->ijab", mij, tau)
             - es("cb,ijac->ijab", mab, t2) - 0.5 * es("bd,ijad->ijab", mvv, tau) + 0.5 * tau + 0.5 * l2)
    gOvvO = es("kiac,jc,kb->iabj", l2, t1, t1) + pvOOv.transpose(1, 0, 3, 2)
    govVO = es("ia,jb->iabj", l1, t1) - es("ikac,jc,kb->iabj", l2, t1, t1) + pvoOV.transpose(1, 0, 3, 2)
    dovvo = 2 * govVO + gOvvO
    doovv = (-2 * gOvvO - govVO).transpose(3, 0, 1, 2)
    tau_h = tau - 0.5 * t2
    goovv = (goovv + es("dlib,jlda->ijab", pvOOv, tau_h) - es("dlia,jldb->ijab", pvoOV, tau_h)
             + es("dlia,jlbd->ijab", pvoOV + 0.5 * pvOOv, t2))
    dovov = 2 * goovv.transpose(0, 2, 1, 3) - goovv.transpose(1, 2, 0, 3)
    gvvvv = es("ijab,ijcd->abcd", l2, t2) + es("ijab,ic,jd->abcd", l2, t1, t1)
    dvvvv = gvvvv.transpose(0, 2, 1, 3) - 0.5 * gvvvv.transpose(0, 3, 1, 2)
    gvovv = (-es("adbc,id->aibc", gvvvv, t1) + es("akic,kb->aibc", pvoOV, t1) - es("akib,kc->aibc", pvOOv, t1)
             + es("ja,jibc->aibc", l1, t2) + es("ja,jb,ic->aibc", l1, t1, t1) + 0.5 * es("ba,ic->aibc", mvv, t1)
             + es("ja,jibc->aibc", t1, l2))
    dovvv = 2 * gvovv.transpose(1, 3, 0, 2) - gvovv.transpose(1, 2, 0, 3)
    return dovov, dvvvv, doooo, doovv, dovvo, None, dovvv, dooov


def rdm2_mo(d2):
    """Full MO 2-RDM (chemist order) from the gamma2 blocks."""
    dovov, dvvvv, doooo, doovv, dovvo, _, dovvv, dooov = d2
    nocc, nvir = dovov.shape[:2]
    n = nocc + nvir
    o, v = slice(0, nocc), slice(nocc, n)
    dm2 = np.zeros((n,) * 4)
    dm2[o, v, o, v] = dovov + dovov.transpose(2, 3, 0, 1)
    dm2[v, o, v, o] = dm2[o, v, o, v].transpose(1, 0, 3, 2)
    dm2[o, o, v, v] = doovv + doovv.transpose(1, 0, 3, 2)
    dm2[v, v, o, o] = dm2[o, o, v, v].transpose(2, 3, 0, 1)
    dm2[o, v, v, o] = dovvo + dovvo.transpose(3, 2, 1, 0)
    dm2[v, o, o, v] = dm2[o, v, v, o].transpose(1, 0, 3, 2)
    dm2[v, v, v, v] = 2 * (dvvvv + dvvvv.transpose(1, 0, 3, 2))
    dm2[o, o, o, o] = 2 * (doooo + doooo.transpose(1, 0, 3, 2))
    dm2[o, v, v, v] = dovvv
    dm2[v, v, o, v] = dovvv.transpose(2, 3, 0, 1)
    dm2[v, v, v, o] = dovvv.transpose(3, 2, 1, 0)
    dm2[v, o, v, v] = dovvv.transpose(1, 0, 3, 2)
    dm2[o, o, o, v] = dooov
    dm2[o, v, o, o] = dooov.transpose(2, 3, 0, 1)
    dm2[o, o, v, o] = dooov.transpose(1, 0, 3, 2)
    dm2[v, o, o, o] = dooov.transpose(3, 2, 1, 0)
    return dm2.transpose(1, 0, 3, 2)


def rdm2_mo2ao_tril(d2, mo_coeff):
    """MO -> AO, (pq) and (rs) symmetrised, lower-triangle packed (nao_pair, nao_pair)."""
    dm2 = es("pi,qj,rk,sl,ijkl->pqrs", mo_coeff, mo_coeff, mo_coeff, mo_coeff, rdm2_mo(d2))
    dm2 = dm2 + dm2.transpose(1, 0, 2, 3)
    dm2 = 0.5 * (dm2 + dm2.transpose(0, 1, 3, 2))
    nao = mo_coeff.shape[0]
    r, c = np.tril_indices(nao)
    p = r * nao + c
    return dm2.reshape(nao * nao, nao * nao)[p[:, None], p[None, :]]
