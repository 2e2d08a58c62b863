"""The chemistry oracle pinned by mathematics (CPU): two-electron FCI, finite
differences of the CCSD energy, integral identities."""
import numpy as np

from ccsd_gpu_b200.gto import M
from oracle import int1e_oracle as O
from oracle import scf_cc_oracle as Q


def test_ccsd_equals_fci_for_two_electrons():
    mf = Q.rhf(M(atom="H 0 0 0; H 0 0 0.74", basis="cc-pvdz"))
    e, _, _ = Q.ccsd(Q.mo_eris(mf))
    assert abs(mf.e_tot + e - Q.fci_2e(mf)) < 1e-10


def test_one_electron_derivative_identities():
    mol = M(atom="O 0 0 0; H 0 -0.757 0.587; H 0 0.757 0.587", basis="cc-pvdz")
    s1 = O.int1e(mol, "int1e_ipovlp")
    t1 = O.int1e(mol, "int1e_ipkin")
    assert np.abs(s1 + s1.transpose(0, 2, 1)).max() < 1e-13   # <d mu|nu> = -<mu|d nu>
    assert np.abs(t1 + t1.transpose(0, 2, 1)).max() < 1e-12


def test_ccsd_gradient_matches_finite_differences():
    mol = M(atom="O 0 0 0; H 0 -0.757 0.587; H 0.05 0.757 0.587", basis="sto-3g")
    _, g = Q.ccsd_gradient(mol)
    assert np.abs(g.sum(0)).max() < 1e-10                      # translational invariance
    x0 = mol.atom_coords()
    h = 1e-3
    for a, x in [(0, 2), (1, 1), (2, 0)]:
        e = []
        for s in (1, -1):
            xx = x0.copy()
            xx[a, x] += s * h
            e.append(Q.ccsd_total(mol.copy().set_geom_(xx))[2])
        assert abs((e[0] - e[1]) / (2 * h) - g[a, x]) < 5e-7
