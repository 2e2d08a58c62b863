"""ORACLE -- test infrastructure only.

One-electron integrals by the McMurchie-Davidson method (Hermite expansion
coefficients E and Hermite Coulomb integrals R over the Boys function), a
different route from the Obara-Saika / Rys recurrences of the CUDA kernel.
Conventions of libcint (as PySCF's mol.intor): coefficients from _env,
angular factor for s and p, "ip" = d/dr on the first function.
Used for int1e_ovlp, int1e_kin, int1e_nuc, int1e_rinv and their ip forms.
"""
from math import pi, sqrt

import numpy as np

from . import eri as _eri


def _cart(l):
    return [(a, b, l - a - b) for a in range(l, -1, -1) for b in range(l - a, -1, -1)]


def _E(i, j, t, Qx, a, b):
    """Hermite expansion coefficient E^{ij}_t (recursive definition)."""
    p = a + b
    q = a * b / p
    if t < 0 or t > i + j:
        return 0.0
    if i == j == t == 0:
        return np.exp(-q * Qx * Qx)
    if j == 0:
        return (1 / (2 * p)) * _E(i - 1, j, t - 1, Qx, a, b) - (q * Qx / a) * _E(i - 1, j, t, Qx, a, b) \
            + (t + 1) * _E(i - 1, j, t + 1, Qx, a, b)
    return (1 / (2 * p)) * _E(i, j - 1, t - 1, Qx, a, b) + (q * Qx / b) * _E(i, j - 1, t, Qx, a, b) \
        + (t + 1) * _E(i, j - 1, t + 1, Qx, a, b)


def _R(t, u, v, n, p, PC, F):
    """Hermite Coulomb integral R^n_{tuv}."""
    if t < 0 or u < 0 or v < 0:
        return 0.0
    if t == u == v == 0:
        return (-2 * p) ** n * F[n]
    if t == u == 0:
        return (v - 1) * _R(t, u, v - 2, n + 1, p, PC, F) + PC[2] * _R(t, u, v - 1, n + 1, p, PC, F)
    if t == 0:
        return (u - 1) * _R(t, u - 2, v, n + 1, p, PC, F) + PC[1] * _R(t, u - 1, v, n + 1, p, PC, F)
    return (t - 1) * _R(t - 2, u, v, n + 1, p, PC, F) + PC[0] * _R(t - 1, u, v, n + 1, p, PC, F)


def _prim(kind, la, lb, a, b, A, B, C=None):
    """Primitive integral between x^la-type monomials (tuples) at A, B."""
    p = a + b
    P = (a * np.asarray(A) + b * np.asarray(B)) / p
    Q = np.asarray(A) - np.asarray(B)
    if kind == "ovlp":
        return np.prod([_E(la[x], lb[x], 0, Q[x], a, b) for x in range(3)]) * (pi / p) ** 1.5
    if kind == "kin":
        def s(lbx):
            return _prim("ovlp", la, lbx, a, b, A, B)
        tot = 0.0
        for x in range(3):
            l = list(lb)
            jb = l[x]
            term = -2 * b * (2 * jb + 1) * s(tuple(l))
            l2 = list(lb); l2[x] += 2
            term += 4 * b * b * s(tuple(l2))
            if jb > 1:
                l3 = list(lb); l3[x] -= 2
                term += jb * (jb - 1) * s(tuple(l3))
            tot += -0.5 * term
        return tot
    # 1/|r - C|
    PC = P - np.asarray(C)
    L = sum(la) + sum(lb)
    F = _eri.boys(L, p * float(PC @ PC))
    tot = 0.0
    for t in range(la[0] + lb[0] + 1):
        Ex = _E(la[0], lb[0], t, Q[0], a, b)
        for u in range(la[1] + lb[1] + 1):
            Ey = _E(la[1], lb[1], u, Q[1], a, b)
            for v in range(la[2] + lb[2] + 1):
                tot += Ex * Ey * _E(la[2], lb[2], v, Q[2], a, b) * _R(t, u, v, 0, p, PC, F)
    return 2 * pi / p * tot


def _cfac(l):
    return 0.282094791773878143 if l == 0 else (0.488602511902919921 if l == 1 else 1.0)


def int1e_cart(mol, name, origin_atom=None):
    """Cartesian (ncomp, nao, nao) matrix for the molecule (nctr-aware)."""
    deriv = name.startswith("int1e_ip")
    kind = {"ovlp": "ovlp", "kin": "kin", "nuc": "nuc", "rinv": "rinv"}[name.split("_ip")[-1].split("int1e_")[-1]]
    atm, bas, env = mol._atm, mol._bas, mol._env
    ao = mol.ao_loc_nr(cart=True)
    nao = ao[-1]
    out = np.zeros((3 if deriv else 1, nao, nao))
    coords = mol.atom_coords()
    charges = mol.atom_charges()
    if kind == "nuc":
        centers = [(coords[c], -float(charges[c])) for c in range(mol.natm)]
    elif kind == "rinv":
        centers = [(coords[origin_atom], 1.0)]
    for ish in range(mol.nbas):
        li, npi, nci = bas[ish, 1], bas[ish, 2], bas[ish, 3]
        ai = env[bas[ish, 5]:bas[ish, 5] + npi]
        ci = env[bas[ish, 6]:bas[ish, 6] + npi * nci].reshape(nci, npi)
        A = coords[bas[ish, 0]]
        for jsh in range(mol.nbas):
            lj, npj, ncj = bas[jsh, 1], bas[jsh, 2], bas[jsh, 3]
            aj = env[bas[jsh, 5]:bas[jsh, 5] + npj]
            cj = env[bas[jsh, 6]:bas[jsh, 6] + npj * ncj].reshape(ncj, npj)
            B = coords[bas[jsh, 0]]
            fac = _cfac(li) * _cfac(lj)
            for fi, mi in enumerate(_cart(li)):
                for fj, mj in enumerate(_cart(lj)):
                    prim = np.zeros((3 if deriv else 1, npi, npj))
                    for p_ in range(npi):
                        for q_ in range(npj):
                            a, b = ai[p_], aj[q_]

                            def ev(la):
                                if kind in ("ovlp", "kin"):
                                    return _prim(kind, la, mj, a, b, A, B)
                                return sum(z * _prim("v", la, mj, a, b, A, B, C) for C, z in centers)
                            if not deriv:
                                prim[0, p_, q_] = ev(mi)
                            else:
                                for x in range(3):
                                    up = list(mi); up[x] += 1
                                    val = -2 * a * ev(tuple(up))
                                    if mi[x] > 0:
                                        dn = list(mi); dn[x] -= 1
                                        val += mi[x] * ev(tuple(dn))
                                    prim[x, p_, q_] = val
                    for c1 in range(nci):
                        for c2 in range(ncj):
                            i = ao[ish] + c1 * len(_cart(li)) + fi
                            j = ao[jsh] + c2 * len(_cart(lj)) + fj
                            out[:, i, j] = fac * np.einsum("p,xpq,q->x", ci[c1], prim, cj[c2])
    return out


def int1e(mol, name, origin_atom=None):
    """Matrix in the molecule's native basis: (nao, nao) or (3, nao, nao)."""
    out = int1e_cart(mol, name, origin_atom)
    if not mol.cart:
        C = mol.cart2sph_coeff()
        out = np.einsum("pi,xpq,qj->xij", C, out, C)
    return out if name.startswith("int1e_ip") else out[0]
