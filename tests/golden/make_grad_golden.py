"""Regenerate the golden CCSD-gradient fixture by running the REFERENCE's own
``grad_elec_gpu`` (ccsd_gpu/gpu_ccsd_grad.py:344-586) on the CPU.

The reference imports cupy and pyscf, neither of which is installed here.  On
top of the stand-ins of make_cc_golden.py (cupy -> numpy, pyscf.lib helpers),
the PySCF pieces the gradient assembly calls are restated from their published
definitions, backed by the oracle:
  * ``mol.intor("int2e" / "int2e_ip1", aosym="s2kl", shls_slice=...)`` -- the
    reference's own ERI kernels compiled for the CPU (oracle/_ref, built by
    oracle/build_ref.py), spherical through the cart2sph matrix;
  * ``mf.get_veff`` = J - K/2 from the full ERI tensor, ``mf.make_rdm1``,
    ``mf.get_ovlp``;
  * ``nuc_grad_method().hcore_generator`` / ``get_ovlp`` / ``grad_nuc``
    (pyscf.grad.rhf) from the McMurchie-Davidson one-electron oracle;
  * ``rhf_grad.make_rdm1e`` = sum_i 2 e_i C_i C_i^T;
  * ``cphf.solve``: (e_a - e_i) x + fvind(x) = -Xvo, solved exactly (PySCF
    iterates the same equation to 1e-9 with a Krylov solver);
  * ``pyscf.grad.mp2._shell_prange`` / ``_index_frozen_active`` /
    ``has_frozen_orbitals``.
Inputs: H2O/cc-pVDZ at the benchmark geometry (O at the origin, H at
(0, +-0.757, 0.587) A), SCF, CCSD and Lambda from the oracle
(oracle/scf_cc_oracle.py); once with all electrons and once with the O 1s
orbital frozen.  The fixture stores the orbitals, the amplitudes and the
reference's electronic gradient, so the GPU path and the oracle can be
checked against the reference's own assembly on identical inputs.

Run from the repository root (needs oracle/_ref, see oracle/build_ref.py):
    python tests/golden/make_grad_golden.py <reference checkout>   (or set REF_ROOT)
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import make_cc_golden as MC  # noqa: E402
from oracle import cc_oracle as C  # noqa: E402
from oracle import eri as E  # noqa: E402
from oracle import int1e_oracle as O  # noqa: E402
from oracle import scf_cc_oracle as Q  # noqa: E402
from ccsd_gpu_b200.gto import M  # noqa: E402

OUT = os.path.join(HERE, "grad_h2o_ccpvdz.npz")
H2O = "O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587"


def _extend_stubs():
    lib = sys.modules["pyscf.lib"]
    lib.direct_sum = lambda spec, a, b: a[:, None] + b[None, :]       # only "i+j->ij" is used
    cphf = sys.modules["pyscf.scf.cphf"]

    def solve(fvind, mo_energy, mo_occ, h1, max_cycle=20, tol=1e-9, **kw):
        occ = mo_occ > 0
        e_ai = mo_energy[~occ][:, None] - mo_energy[occ][None, :]
        n = h1.size
        A = np.zeros((n, n))
        for k in range(n):
            x = np.zeros(n)
            x[k] = 1.0
            A[:, k] = np.asarray(fvind(x.reshape(h1.shape))).ravel()
        A += np.diag(e_ai.ravel())
        return np.linalg.solve(A, -h1.ravel()).reshape(h1.shape), None
    cphf.solve = solve
    rg = sys.modules["pyscf.grad.rhf"]

    def make_rdm1e(mo_energy, mo_coeff, mo_occ):
        occ = mo_occ > 0
        c = mo_coeff[:, occ]
        return (c * (mo_energy * mo_occ)[occ]) @ c.T
    rg.make_rdm1e = make_rdm1e
    mp2 = sys.modules["pyscf.grad.mp2"]

    def _shell_prange(mol, start, stop, blksize):
        ao = mol.ao_loc_nr()
        b0 = start
        for b in range(start, stop):
            if ao[b + 1] - ao[b0] > blksize and b > b0:
                yield b0, b, int(ao[b] - ao[b0])
                b0 = b
        yield b0, stop, int(ao[stop] - ao[b0])
    mp2._shell_prange = _shell_prange

    def _index_frozen_active(mask, mo_occ):
        occ = mo_occ > 0
        return (np.where(mask & occ)[0], np.where(mask & ~occ)[0], np.where(~mask & occ)[0],
                np.where(~mask & ~occ)[0])
    mp2._index_frozen_active = _index_frozen_active
    mp2.has_frozen_orbitals = lambda mycc: not mycc.get_frozen_mask().all()


class _Mol:
    """The molecule plus the ``intor`` calls the gradient assembly makes."""

    def __init__(self, mol):
        self._m = mol

    def __getattr__(self, name):
        return getattr(self._m, name)

    def intor(self, name, comp=None, aosym="s1", shls_slice=None):
        assert aosym == "s2kl" and shls_slice is not None
        b0, b1 = shls_slice[:2]
        assert tuple(shls_slice[2:]) == (0, self._m.nbas) * 3
        impl = "ref" if E.ref_available() else "oracle"
        return E.s2kl(self._m, b0, b1, 1 if name == "int2e_ip1" else 0, impl=impl)


def _scf_like(mol, mf):
    eri = mf.eri

    class GradRHF:
        def hcore_generator(self, m=None):
            h1 = -(O.int1e(mol, "int1e_ipkin") + O.int1e(mol, "int1e_ipnuc"))
            off = mol.offset_nr_by_atom()

            def hcore_deriv(a):
                p0, p1 = int(off[a, 2]), int(off[a, 3])
                v = -mol.atom_charges()[a] * O.int1e(mol, "int1e_iprinv", origin_atom=a)
                v[:, p0:p1] += h1[:, p0:p1]
                return v + v.transpose(0, 2, 1)
            return hcore_deriv

        def get_ovlp(self, m=None):
            return -O.int1e(mol, "int1e_ipovlp")

        def grad_nuc(self):
            return mol.grad_nuc()

    return types.SimpleNamespace(
        mol=mol, mo_energy=mf.mo_energy, mo_coeff=mf.mo_coeff, mo_occ=mf.mo_occ,
        make_rdm1=lambda c, o: (c * o) @ c.T, get_ovlp=lambda *a: mf.S,
        get_veff=lambda m=None, dm=None: Q.veff(eri, dm), nuc_grad_method=lambda: GradRHF())


def frozen_state(mf, nfrozen):
    """CCSD + Lambda in the active space (the lowest nfrozen orbitals frozen;
    Fock matrix of the full HF density)."""
    eris = Q.mo_eris(mf)
    if nfrozen:
        g = eris.g[nfrozen:, nfrozen:, nfrozen:, nfrozen:]
        fock = eris.fock[nfrozen:, nfrozen:]
        nocc = eris.nocc - nfrozen
        eris = types.SimpleNamespace(fock=fock, mo_energy=np.diag(fock).copy(), nocc=nocc, g=g,
                                     **vars(C.mo_blocks(g, nocc)))
    _, t1, t2 = Q.ccsd(eris)
    l1, l2 = Q.lambda_solve(t1, t2, eris)
    return t1, t2, l1, l2


def main():
    REF = MC.ref_root()
    MC._stub_modules()
    _extend_stubs()
    grd = MC._load("ref_gpu_ccsd_grad", os.path.join(REF, "ccsd_gpu", "gpu_ccsd_grad.py"))
    mol = M(atom=H2O, basis="cc-pvdz")
    mf = Q.rhf(mol)
    out = dict(atom=np.array(H2O), basis=np.array("cc-pvdz"), mo_coeff=mf.mo_coeff, mo_energy=mf.mo_energy,
               mo_occ=mf.mo_occ, e_hf=mf.e_tot, grad_nuc=mol.grad_nuc())
    for nfrozen in (0, 1):
        t1, t2, l1, l2 = frozen_state(mf, nfrozen)
        mask = np.ones(len(mf.mo_energy), dtype=bool)
        mask[:nfrozen] = False
        mycc = types.SimpleNamespace(
            mol=_Mol(mol), mo_coeff=mf.mo_coeff, mo_occ=mf.mo_occ, _scf=_scf_like(mol, mf), max_memory=1e6,
            stdout=None, verbose=0, get_frozen_mask=lambda mask=mask: mask)
        de = grd.grad_elec_gpu(mycc, t1, t2, l1, l2, verbose=0)
        tag = "fc%d" % nfrozen
        out.update({tag + "_t1": t1, tag + "_t2": t2, tag + "_l1": l1, tag + "_l2": l2, tag + "_de": de})
        print(tag, "reference grad_elec_gpu:\n", de)
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
