"""Molecule container with PySCF's ``_atm`` / ``_bas`` / ``_env`` layout.

The integral entry points of the reference take a ``pyscf.gto.Mole`` and read
``mol._atm``, ``mol._bas``, ``mol._env``, ``mol.cart``, ``mol.nbas``,
``mol.ao_loc_nr()``, ``mol.cart2sph_coeff()`` and ``mol.copy()``
(ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216, 223-289, 320-326).  PySCF is
not a dependency of this package, so :class:`Mole` provides exactly that
surface (plus what the gradient driver reads: ``offset_nr_by_atom``,
``atom_coords``, ``atom_charges``, ``energy_nuc``, ``nelectron``).  A real
PySCF ``Mole`` is accepted everywhere a :class:`Mole` is.

Conventions restated from PySCF 2.12 / libcint 6:
  * slots: ``_atm`` rows ``[Z, ptr_coord, nuc_mod, ptr_zeta, 0, 0]``;
    ``_bas`` rows ``[atom, l, nprim, nctr, kappa, ptr_exp, ptr_coeff, 0]``;
    ``_env[:20]`` is reserved (PTR_ENV_START = 20);
  * contraction coefficients in ``_env`` carry the radial normalisation
    ``gto_norm(l, a) = 1/sqrt(int_0^inf r^(2l+2) exp(-2 a r^2) dr)`` and each
    contracted radial function is normalised to one;
  * coefficient of contraction c, primitive p sits at ``ptr_coeff + c*nprim + p``;
  * AO order: atoms in input order, shells in basis order, within a shell
    contraction-major then component (Cartesian lexicographic, or real
    spherical m = -l..l, with p as x, y, z).
"""
import copy as _copy
import math

import numpy as np

from . import basis_data
from .cart2sph import cart2sph_block

BOHR = 0.52917721092          # Angstrom per bohr, PySCF's lib.param.BOHR
PTR_ENV_START = 20
ATM_SLOTS = 6
BAS_SLOTS = 8
CHARGE_OF, PTR_COORD, NUC_MOD_OF, PTR_ZETA = 0, 1, 2, 3
ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, KAPPA_OF, PTR_EXP, PTR_COEFF = 0, 1, 2, 3, 4, 5, 6

_ELEMENTS = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
             "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar"]
CHARGE = {s: z for z, s in enumerate(_ELEMENTS) if z > 0}


def gaussian_int(n, alpha):
    """int_0^inf x^n exp(-alpha x^2) dx."""
    n1 = (n + 1) * 0.5
    return math.gamma(n1) / (2.0 * np.asarray(alpha, dtype=np.float64) ** n1)


def gto_norm(l, expnt):
    """Radial normalisation of r^l exp(-a r^2)."""
    return 1.0 / np.sqrt(gaussian_int(2 * l + 2, 2 * np.asarray(expnt, dtype=np.float64)))


def normalized_coefficients(l, exps, coefs):
    """(nprim, nctr) coefficients as stored in ``_env`` for one shell."""
    es = np.asarray(exps, dtype=np.float64)
    cs = np.asarray(coefs, dtype=np.float64).reshape(len(es), -1)
    cs = cs * gto_norm(l, es)[:, None]
    ee = gaussian_int(2 * l + 2, es[:, None] + es[None, :])
    s1 = 1.0 / np.sqrt(np.einsum("pi,pq,qi->i", cs, ee, cs))
    return cs * s1[None, :]


def parse_atoms(atom, unit="angstrom"):
    if isinstance(atom, str):
        rows = []
        for item in atom.replace(";", "\n").splitlines():
            parts = item.split()
            if not parts:
                continue
            rows.append((parts[0], tuple(float(v) for v in parts[1:4])))
    else:
        rows = [(a[0], tuple(float(v) for v in a[1])) for a in atom]
    scale = 1.0 / BOHR if unit.lower().startswith("a") else 1.0
    out = []
    for sym, xyz in rows:
        sym = sym.strip()
        sym = sym[0].upper() + sym[1:].lower()
        if sym not in CHARGE:
            raise KeyError("unknown element %r" % sym)
        out.append((sym, np.array(xyz, dtype=np.float64) * scale))
    return out


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nsph(l):
    return 2 * l + 1


class Mole:
    """Minimal PySCF-compatible molecule: geometry, basis, integral layout."""

    def __init__(self, atom=None, basis="cc-pvdz", unit="angstrom", charge=0, spin=0,
                 cart=False, verbose=0):
        self.atom = atom
        self.basis = basis
        self.unit = unit
        self.charge = charge
        self.spin = spin
        self.cart = cart
        self.verbose = verbose
        self.max_memory = 16000
        if atom is not None:
            self.build()

    # -- construction -----------------------------------------------------
    def build(self):
        atoms = parse_atoms(self.atom, self.unit)
        self._atom = atoms
        env = [0.0] * PTR_ENV_START
        atm = []
        for sym, xyz in atoms:
            ptr = len(env)
            env.extend(xyz.tolist())
            env.append(0.0)              # nuclear model zeta (point nucleus)
            atm.append([CHARGE[sym], ptr, 1, ptr + 3, 0, 0])
        bas = []
        basis_ptr = {}
        for ia, (sym, _) in enumerate(atoms):
            bname = self.basis[sym] if isinstance(self.basis, dict) else self.basis
            if sym not in basis_ptr:
                shells = []
                for shell in basis_data.load(bname, sym):
                    l = shell[0]
                    rows = np.array(shell[1:], dtype=np.float64)
                    es, cs = rows[:, 0], rows[:, 1:]
                    cs = normalized_coefficients(l, es, cs)
                    pexp = len(env)
                    env.extend(es.tolist())
                    pcoef = len(env)
                    env.extend(cs.T.ravel().tolist())
                    shells.append((l, len(es), cs.shape[1], pexp, pcoef))
                basis_ptr[sym] = shells
            for l, nprim, nctr, pexp, pcoef in basis_ptr[sym]:
                bas.append([ia, l, nprim, nctr, 0, pexp, pcoef, 0])
        self._atm = np.asarray(atm, dtype=np.int32).reshape(-1, ATM_SLOTS)
        self._bas = np.asarray(bas, dtype=np.int32).reshape(-1, BAS_SLOTS)
        self._env = np.asarray(env, dtype=np.float64)
        return self

    def copy(self):
        new = _copy.copy(self)
        new._atm = self._atm.copy()
        new._bas = self._bas.copy()
        new._env = self._env.copy()
        return new

    def set_geom_(self, coords_bohr):
        """Replace the nuclear coordinates (bohr) in place; basis layout unchanged."""
        coords_bohr = np.asarray(coords_bohr, dtype=np.float64).reshape(self.natm, 3)
        for ia in range(self.natm):
            p = self._atm[ia, PTR_COORD]
            self._env[p:p + 3] = coords_bohr[ia]
        return self

    # -- sizes ----------------------------------------------------------------
    @property
    def natm(self):
        return len(self._atm)

    @property
    def nbas(self):
        return len(self._bas)

    @property
    def nelectron(self):
        return int(self._atm[:, CHARGE_OF].sum()) - self.charge

    @property
    def nao(self):
        return self.nao_nr()

    def nao_nr(self, cart=None):
        return int(self.ao_loc_nr(cart)[-1])

    def nao_cart(self):
        return self.nao_nr(cart=True)

    def ao_loc_nr(self, cart=None):
        if cart is None:
            cart = self.cart
        l = self._bas[:, ANG_OF]
        nctr = self._bas[:, NCTR_OF]
        dims = ((l + 1) * (l + 2) // 2 if cart else 2 * l + 1) * nctr
        loc = np.zeros(self.nbas + 1, dtype=np.int32)
        np.cumsum(dims, out=loc[1:])
        return loc

    # -- geometry -------------------------------------------------------------
    def atom_coords(self, unit="bohr"):
        ptr = self._atm[:, PTR_COORD]
        c = self._env[np.stack([ptr, ptr + 1, ptr + 2], axis=1)]
        return c * BOHR if unit.lower().startswith("a") else c

    def atom_charges(self):
        return self._atm[:, CHARGE_OF].astype(np.int64)

    def atom_symbol(self, ia):
        return self._atom[ia][0]

    def energy_nuc(self):
        z = self.atom_charges().astype(np.float64)
        r = self.atom_coords()
        e = 0.0
        for i in range(self.natm):
            for j in range(i):
                e += z[i] * z[j] / np.linalg.norm(r[i] - r[j])
        return e

    def grad_nuc(self):
        """d E_nuc / d R  (natm, 3)."""
        z = self.atom_charges().astype(np.float64)
        r = self.atom_coords()
        g = np.zeros((self.natm, 3))
        for i in range(self.natm):
            for j in range(self.natm):
                if i != j:
                    d = r[i] - r[j]
                    g[i] -= z[i] * z[j] * d / np.linalg.norm(d) ** 3
        return g

    def offset_nr_by_atom(self):
        """Rows (shell0, shell1, ao0, ao1) per atom."""
        ao_loc = self.ao_loc_nr()
        out = np.zeros((self.natm, 4), dtype=np.int64)
        for ia in range(self.natm):
            sh = np.where(self._bas[:, ATOM_OF] == ia)[0]
            s0, s1 = (int(sh[0]), int(sh[-1]) + 1) if len(sh) else (0, 0)
            out[ia] = (s0, s1, ao_loc[s0], ao_loc[s1])
        return out

    def cart2sph_coeff(self):
        """(nao_cart, nao_sph) block-diagonal matrix: sph_ao = cart_ao @ C."""
        lc = self.ao_loc_nr(cart=True)
        ls = self.ao_loc_nr(cart=False)
        C = np.zeros((lc[-1], ls[-1]))
        for ib in range(self.nbas):
            l = int(self._bas[ib, ANG_OF])
            blk = cart2sph_block(l)
            nc, ns = blk.shape
            for c in range(int(self._bas[ib, NCTR_OF])):
                r0 = lc[ib] + c * nc
                c0 = ls[ib] + c * ns
                C[r0:r0 + nc, c0:c0 + ns] = blk
        return C


def M(**kwargs):
    """``gto.M``-style constructor."""
    return Mole(**kwargs)
