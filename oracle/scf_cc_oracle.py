"""ORACLE -- test infrastructure only.

numpy restatements of the supporting chemistry around the reference's hot
path, for small molecules:
  * rhf(mol): closed-shell Hartree-Fock with DIIS (PySCF scf.RHF, which the
    reference's driver runs on the CPU: examples/h2o_ccsd_grad.py:118-121);
  * ccsd(...): RCCSD T amplitudes, the equations of PySCF's rccsd.update_amps
    and rintermediates (the reference delegates them to gpu4pyscf/PySCF:
    examples/h2o_ccsd_grad.py:128-147);
  * fci_2e(...): exact two-electron energy (CCSD is exact for two electrons);
  * grad_elec(...): the CCSD nuclear gradient exactly as the reference's
    grad_elec_gpu assembles it (ref: ccsd_gpu/gpu_ccsd_grad.py:344-586), with
    full tensors and an exact CPHF solve;
ERIs come from the C oracle (eri_oracle.c), one-electron integrals from the
McMurchie-Davidson oracle (int1e_oracle.py).
"""
from types import SimpleNamespace

import numpy as np

from . import cc_oracle as C
from . import eri as E
from . import int1e_oracle as O

es = C.es


def full_eri(mol):
    """(nao,)*4 chemist-notation ERIs in the native basis."""
    s2kl = E.s2kl(mol, 0, mol.nbas, 0)
    n = s2kl.shape[1]
    k, l = np.tril_indices(n)
    g = np.zeros((n, n, n, n))
    g[:, :, k, l] = s2kl
    g[:, :, l, k] = s2kl
    return g


def full_eri_ip1(mol):
    """(3, nao, nao, nao, nao): (d/dr_1 i j|kl)."""
    s2kl = E.s2kl(mol, 0, mol.nbas, 1)
    n = s2kl.shape[2]
    k, l = np.tril_indices(n)
    g = np.zeros((3, n, n, n, n))
    g[..., k, l] = s2kl
    g[..., l, k] = s2kl
    return g


def jk(eri, dm):
    return es("pqrs,rs->pq", eri, dm), es("prqs,rs->pq", eri, dm)


def veff(eri, dm):
    J, K = jk(eri, dm)
    return J - 0.5 * K


def rhf(mol, eri=None, conv=1e-11, max_cycle=100):
    S = O.int1e(mol, "int1e_ovlp")
    h = O.int1e(mol, "int1e_kin") + O.int1e(mol, "int1e_nuc")
    eri = full_eri(mol) if eri is None else eri
    nocc = mol.nelectron // 2
    w, U = np.linalg.eigh(S)
    X = U / np.sqrt(w)
    e, Cp = np.linalg.eigh(X.T @ h @ X)
    Cm = X @ Cp
    dm = 2 * Cm[:, :nocc] @ Cm[:, :nocc].T
    fs, errs = [], []
    e_old = 0.0
    for it in range(max_cycle):
        F = h + veff(eri, dm)
        err = F @ dm @ S - S @ dm @ F
        fs.append(F); errs.append(err)
        fs, errs = fs[-8:], errs[-8:]
        n = len(fs)
        if n > 1:
            B = -np.ones((n + 1, n + 1)); B[n, n] = 0
            for i in range(n):
                for j in range(n):
                    B[i, j] = np.vdot(errs[i], errs[j])
            rhs = np.zeros(n + 1); rhs[n] = -1
            c = np.linalg.solve(B, rhs)[:n]
            F = sum(ci * fi for ci, fi in zip(c, fs))
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        Cm = X @ Cp
        dm_new = 2 * Cm[:, :nocc] @ Cm[:, :nocc].T
        Fn = h + veff(eri, dm_new)
        etot = 0.5 * np.sum(dm_new * (h + Fn)) + mol.energy_nuc()
        done = abs(etot - e_old) < conv and np.abs(dm_new - dm).max() < 1e-8
        dm, e_old = dm_new, etot
        if done:
            break
    F = h + veff(eri, dm)
    e, Cp = np.linalg.eigh(X.T @ F @ X)
    Cm = X @ Cp
    occ = np.zeros(len(e)); occ[:nocc] = 2
    return SimpleNamespace(mol=mol, mo_energy=e, mo_coeff=Cm, mo_occ=occ, e_tot=etot, S=S, h=h, eri=eri,
                           converged=done)


def mo_eris(mf):
    """PySCF-style eris (fock, mo_energy and chemist blocks) of an RHF solution."""
    Cm = mf.mo_coeff
    g = es("pi,qj,rk,sl,pqrs->ijkl", Cm, Cm, Cm, Cm, mf.eri)
    nocc = int((mf.mo_occ > 0).sum())
    dm = 2 * Cm[:, :nocc] @ Cm[:, :nocc].T
    fock = Cm.T @ (mf.h + veff(mf.eri, dm)) @ Cm
    blocks = C.mo_blocks(g, nocc)
    return SimpleNamespace(fock=fock, mo_energy=np.diag(fock).copy(), nocc=nocc, g=g, **vars(blocks))


def ccsd_update(t1, t2, eris):
    """One Jacobi step of the RCCSD amplitude equations (PySCF rccsd.update_amps)."""
    nocc, nvir = t1.shape
    fock = eris.fock
    foo, fov, fvv = fock[:nocc, :nocc], fock[:nocc, nocc:], fock[nocc:, nocc:]
    eo, ev = eris.mo_energy[:nocc], eris.mo_energy[nocc:]
    ovov, ovvv, ovoo, ovvo, oovv, oooo, vvvv = (eris.ovov, eris.ovvv, eris.ovoo, eris.ovvo, eris.oovv,
                                                eris.oooo, eris.vvvv)
    Foo = foo + 2 * es("kcld,ilcd->ki", ovov, t2) - es("kdlc,ilcd->ki", ovov, t2) \
        + 2 * es("kcld,ic,ld->ki", ovov, t1, t1) - es("kdlc,ic,ld->ki", ovov, t1, t1)
    Fvv = fvv - 2 * es("kcld,klad->ac", ovov, t2) + es("kdlc,klad->ac", ovov, t2) \
        - 2 * es("kcld,ka,ld->ac", ovov, t1, t1) + es("kdlc,ka,ld->ac", ovov, t1, t1)
    Fov = fov + 2 * es("kcld,ld->kc", ovov, t1) - es("kdlc,ld->kc", ovov, t1)
    Loo = Foo + fov @ t1.T + 2 * es("lcki,lc->ki", ovoo, t1) - es("kcli,lc->ki", ovoo, t1)
    Lvv = Fvv - t1.T @ fov + 2 * es("kdac,kd->ac", ovvv, t1) - es("kcad,kd->ac", ovvv, t1)
    Foo = Foo - np.diag(eo)
    Fvv = Fvv - np.diag(ev)
    Loo = Loo - np.diag(eo)
    Lvv = Lvv - np.diag(ev)
    t1n = (-2 * es("kc,ka,ic->ia", fov, t1, t1) + t1 @ Fvv.T - Foo.T @ t1 + 2 * es("kc,kica->ia", Fov, t2)
           - es("kc,ikca->ia", Fov, t2) + es("kc,ic,ka->ia", Fov, t1, t1) + fov
           + 2 * es("kcai,kc->ia", ovvo, t1) - es("kiac,kc->ia", oovv, t1)
           + 2 * es("kdac,ikcd->ia", ovvv, t2) - es("kcad,ikcd->ia", ovvv, t2)
           + 2 * es("kdac,kd,ic->ia", ovvv, t1, t1) - es("kcad,kd,ic->ia", ovvv, t1, t1)
           - 2 * es("lcki,klac->ia", ovoo, t2) + es("kcli,klac->ia", ovoo, t2)
           - 2 * es("lcki,lc,ka->ia", ovoo, t1, t1) + es("kcli,lc,ka->ia", ovoo, t1, t1))
    tmp2 = es("kibc,ka->abic", oovv, -t1) + ovvv.transpose(1, 3, 0, 2)
    tmp = es("abic,jc->ijab", tmp2, t1)
    t2n = tmp + tmp.transpose(1, 0, 3, 2)
    tmp2 = es("kcai,jc->akij", ovvo, t1) + ovoo.transpose(1, 3, 0, 2)
    tmp = es("akij,kb->ijab", tmp2, t1)
    t2n = t2n - tmp - tmp.transpose(1, 0, 3, 2) + ovov.transpose(0, 2, 1, 3)
    Woooo = (es("lcki,jc->klij", ovoo, t1) + es("kclj,ic->klij", ovoo, t1) + es("kcld,ijcd->klij", ovov, t2)
             + es("kcld,ic,jd->klij", ovov, t1, t1) + oooo.transpose(0, 2, 1, 3))
    Wvvvv = -es("kdac,kb->abcd", ovvv, t1) - es("kcbd,ka->abcd", ovvv, t1) + vvvv.transpose(0, 2, 1, 3)
    Wvoov = (es("kcad,id->akic", ovvv, t1) - es("kcli,la->akic", ovoo, t1) + ovvo.transpose(2, 0, 3, 1)
             - 0.5 * es("ldkc,ilda->akic", ovov, t2) - 0.5 * es("lckd,ilad->akic", ovov, t2)
             - es("ldkc,id,la->akic", ovov, t1, t1) + es("ldkc,ilad->akic", ovov, t2))
    Wvovo = (es("kdac,id->akci", ovvv, t1) - es("lcki,la->akci", ovoo, t1) + oovv.transpose(2, 0, 3, 1)
             - 0.5 * es("lckd,ilda->akci", ovov, t2) - es("lckd,id,la->akci", ovov, t1, t1))
    tau = t2 + es("ia,jb->ijab", t1, t1)
    t2n = t2n + es("klij,klab->ijab", Woooo, tau) + es("abcd,ijcd->ijab", Wvvvv, tau)
    tmp = es("ac,ijcb->ijab", Lvv, t2)
    t2n = t2n + tmp + tmp.transpose(1, 0, 3, 2)
    tmp = es("ki,kjab->ijab", Loo, t2)
    t2n = t2n - tmp - tmp.transpose(1, 0, 3, 2)
    tmp = 2 * es("akic,kjcb->ijab", Wvoov, t2) - es("akci,kjcb->ijab", Wvovo, t2)
    t2n = t2n + tmp + tmp.transpose(1, 0, 3, 2)
    tmp = es("akic,kjbc->ijab", Wvoov, t2)
    t2n = t2n - tmp - tmp.transpose(1, 0, 3, 2)
    tmp = es("bkci,kjac->ijab", Wvovo, t2)
    t2n = t2n - tmp - tmp.transpose(1, 0, 3, 2)
    eia = eo[:, None] - ev[None, :]
    return t1n / eia, t2n / (eia[:, None, :, None] + eia[None, :, None, :])


def ccsd_energy(t1, t2, eris):
    nocc = t1.shape[0]
    tau = t2 + es("ia,jb->ijab", t1, t1)
    return (2 * np.sum(eris.fock[:nocc, nocc:] * t1) + 2 * es("ijab,iajb", tau, eris.ovov)
            - es("ijab,ibja", tau, eris.ovov))


def ccsd(eris, tol=1e-11, max_cycle=200):
    nocc = eris.nocc
    eo, ev = eris.mo_energy[:nocc], eris.mo_energy[nocc:]
    eia = eo[:, None] - ev[None, :]
    t1 = eris.fock[:nocc, nocc:] / eia
    t2 = eris.ovov.transpose(0, 2, 1, 3) / (eia[:, None, :, None] + eia[None, :, None, :])
    e_old = ccsd_energy(t1, t2, eris)
    hist = []
    for it in range(max_cycle):
        t1n, t2n = ccsd_update(t1, t2, eris)
        d = np.concatenate([(t1n - t1).ravel(), (t2n - t2).ravel()])
        x = np.concatenate([t1n.ravel(), t2n.ravel()])
        hist.append((x, d))
        hist = hist[-8:]
        if len(hist) > 1:
            n = len(hist)
            B = -np.ones((n + 1, n + 1)); B[n, n] = 0
            for i in range(n):
                for j in range(n):
                    B[i, j] = hist[i][1] @ hist[j][1]
            rhs = np.zeros(n + 1); rhs[n] = -1
            c = np.linalg.solve(B, rhs)[:n]
            x = sum(ci * h[0] for ci, h in zip(c, hist))
        t1, t2 = x[:t1.size].reshape(t1.shape), x[t1.size:].reshape(t2.shape)
        e = ccsd_energy(t1, t2, eris)
        if abs(e - e_old) < tol and np.abs(d).max() < 1e-9:
            break
        e_old = e
    return e, t1, t2


def fci_2e(mf):
    """Exact ground-state energy of a two-electron molecule (singlet, real orbitals)."""
    Cm = mf.mo_coeff
    h = Cm.T @ mf.h @ Cm
    g = es("pi,qj,rk,sl,pqrs->ijkl", Cm, Cm, Cm, Cm, mf.eri)
    n = h.shape[0]
    # Psi = sum_pq c_pq |p_alpha q_beta>,  H c = h c + c h + sum_rs (pr|qs) c_rs
    H = (np.kron(h, np.eye(n)) + np.kron(np.eye(n), h) + g.transpose(0, 2, 1, 3).reshape(n * n, n * n))
    return np.linalg.eigvalsh(H)[0] + mf.mol.energy_nuc()


def grad_elec(mf, t1, t2, l1, l2, eri_ip1=None):
    """CCSD electronic gradient (natm, 3), restating grad_elec_gpu step by step.

    Frozen core orbitals (no frozen virtuals) are taken from the amplitude
    shapes: the RDMs live on the active orbitals and the frozen-active block
    of the relaxed density is Imat / (e_F - e_A) (ref: ccsd_gpu/gpu_ccsd_grad.py:373-378,510-518)."""
    mol = mf.mol
    Cm, e, occ = mf.mo_coeff, mf.mo_energy, mf.mo_occ
    nocc = int((occ > 0).sum())
    nao, nmo = Cm.shape
    nf = nocc - t1.shape[0]
    Ca = Cm[:, nf:]
    eri = mf.eri
    ip1 = full_eri_ip1(mol) if eri_ip1 is None else eri_ip1
    doo, dov, dvo, dvv = C.gamma1(t1, t2, l1, l2)
    d2 = C.gamma2(t1, t2, l1, l2)
    dm2 = es("pi,qj,rk,sl,ijkl->pqrs", Ca, Ca, Ca, Ca, C.rdm2_mo(d2))
    dm2 = dm2 + dm2.transpose(1, 0, 2, 3)
    dm2 = 0.5 * (dm2 + dm2.transpose(0, 1, 3, 2))
    P = 2 * Cm[:, :nocc] @ Cm[:, :nocc].T
    off = mol.offset_nr_by_atom()
    de = np.zeros((mol.natm, 3))
    vhf1 = np.zeros((mol.natm, 3, nao, nao))
    # Imat[p,q] = 1/2 sum (ip|kl) Gamma[iqkl]  (ref: gpu_ccsd_grad.py:443-445 with the s2kl diagonal 1/2)
    Imat = 0.5 * es("ipkl,iqkl->pq", eri, dm2)
    for a in range(mol.natm):
        p0, p1 = int(off[a, 2]), int(off[a, 3])
        I = ip1[:, p0:p1]
        de[a] -= es("xijkl,ijkl->x", I, dm2[p0:p1])
        v = np.zeros((3, nao, nao))
        v += es("xijkl,ij->xkl", I, P[p0:p1])                  # C1
        v -= 0.5 * es("xijkl,il->xkj", I, P[p0:p1])            # X2
        v[:, p0:p1] += es("xijkl,kl->xij", I, P)               # C3
        v[:, p0:p1] -= 0.5 * es("xijkl,jk->xil", I, P)         # X4
        vhf1[a] = v
    S = mf.S
    Imat = Cm.T @ Imat @ S @ Cm * -1
    dm1mo = np.zeros((nmo, nmo))
    dm1mo[nf:nocc, nf:nocc] = doo + doo.T
    dm1mo[nocc:, nocc:] = dvv + dvv.T
    if nf:
        dco = Imat[:nf, nf:nocc] / (e[:nf, None] - e[None, nf:nocc])
        dm1mo[:nf, nf:nocc] = dco
        dm1mo[nf:nocc, :nf] = dco.T
    dm1 = Cm @ dm1mo @ Cm.T
    vhf = veff(eri, dm1) * 2
    Xvo = Cm[:, nocc:].T @ vhf @ Cm[:, :nocc] + Imat[:nocc, nocc:].T - Imat[nocc:, :nocc]
    # CPHF: (e_a - e_i) x + fvind(x) = -Xvo, solved exactly (PySCF solves it to 1e-9)
    nvir = nmo - nocc
    Cv, Co = Cm[:, nocc:], Cm[:, :nocc]
    A = np.zeros((nvir * nocc, nvir * nocc))
    for k in range(nvir * nocc):
        x = np.zeros(nvir * nocc); x[k] = 1
        X = x.reshape(nvir, nocc)
        dm = Cv @ X @ Co.T
        A[:, k] = (Cv.T @ veff(eri, dm + dm.T) @ Co * 2).ravel()
    A += np.diag((e[nocc:, None] - e[None, :nocc]).ravel())
    dvo_z = np.linalg.solve(A, -Xvo.ravel()).reshape(nvir, nocc)
    dm1mo[nocc:, :nocc] += dvo_z
    dm1mo[:nocc, nocc:] += dvo_z.T
    Imat[nocc:, :nocc] = Imat[:nocc, nocc:].T
    im1 = Cm @ Imat @ Cm.T
    s1 = -O.int1e(mol, "int1e_ipovlp")
    h1 = -(O.int1e(mol, "int1e_ipkin") + O.int1e(mol, "int1e_ipnuc"))
    zeta = 0.5 * (e[:, None] + e[None, :])
    zeta[nocc:, :nocc] = e[:nocc]
    zeta[:nocc, nocc:] = e[:nocc].reshape(-1, 1)
    zeta = Cm @ (zeta * dm1mo) @ Cm.T
    dm1 = Cm @ dm1mo @ Cm.T
    p1 = Co @ Co.T
    vhf_s1occ = p1 @ veff(eri, dm1 + dm1.T) @ p1
    dm1p = P + dm1 * 2
    dm1 = dm1 + P
    zeta = zeta + (Co * (e[:nocc] * 2)) @ Co.T
    for a in range(mol.natm):
        p0, p1_ = int(off[a, 2]), int(off[a, 3])
        vr = -mol.atom_charges()[a] * O.int1e(mol, "int1e_iprinv", origin_atom=a)
        vr[:, p0:p1_] += h1[:, p0:p1_]
        h1ao = vr + vr.transpose(0, 2, 1)
        de[a] += es("xij,ij->x", s1[:, p0:p1_], im1[p0:p1_])
        de[a] += es("xji,ij->x", s1[:, p0:p1_], im1[:, p0:p1_])
        de[a] += es("xij,ji->x", h1ao, dm1)
        de[a] -= es("xij,ij->x", s1[:, p0:p1_], zeta[p0:p1_])
        de[a] -= es("xji,ij->x", s1[:, p0:p1_], zeta[:, p0:p1_])
        de[a] -= es("xij,ij->x", s1[:, p0:p1_], vhf_s1occ[p0:p1_]) * 2
        de[a] -= es("xij,ij->x", vhf1[a], dm1p)
    return de


def lambda_solve(t1, t2, eris, tol=1e-11, max_cycle=300):
    imds = C.make_intermediates(t1, t2, eris.fock, eris)
    l1, l2 = t1, t2
    hist = []
    for it in range(max_cycle):
        n1, n2 = C.update_lambda(t1, t2, l1, l2, eris.fock, eris.mo_energy, eris, imds)
        d = np.concatenate([(n1 - l1).ravel(), (n2 - l2).ravel()])
        x = np.concatenate([n1.ravel(), n2.ravel()])
        hist.append((x, d)); hist = hist[-8:]
        if len(hist) > 1:
            n = len(hist)
            B = -np.ones((n + 1, n + 1)); B[n, n] = 0
            for i in range(n):
                for j in range(n):
                    B[i, j] = hist[i][1] @ hist[j][1]
            rhs = np.zeros(n + 1); rhs[n] = -1
            c = np.linalg.solve(B, rhs)[:n]
            x = sum(ci * h[0] for ci, h in zip(c, hist))
        l1, l2 = x[:t1.size].reshape(t1.shape), x[t1.size:].reshape(t2.shape)
        if np.abs(d).max() < tol:
            break
    return l1, l2


def ccsd_total(mol):
    mf = rhf(mol)
    eris = mo_eris(mf)
    ecc, t1, t2 = ccsd(eris)
    return mf, eris, mf.e_tot + ecc, t1, t2


def ccsd_gradient(mol):
    mf, eris, etot, t1, t2 = ccsd_total(mol)
    l1, l2 = lambda_solve(t1, t2, eris)
    return etot, grad_elec(mf, t1, t2, l1, l2) + mol.grad_nuc()
