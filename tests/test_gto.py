"""Host-side data formats: Mole layout, normalisation, cart->sph, decontraction (CPU)."""
import numpy as np

from ccsd_gpu_b200.cuda.basis import _check_mol, decontract_bas, sparse_columns
from ccsd_gpu_b200.gto import M, cart2sph_block, cart_components
from ccsd_gpu_b200.gto.mole import gaussian_int


def test_h2o_ccpvdz_dimensions():
    mol = M(atom="O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587", basis="cc-pvdz")
    assert mol.nao_nr() == 24 and mol.nao_cart() == 25 and mol.nelectron == 10
    assert _check_mol(mol)
    off = mol.offset_nr_by_atom()
    assert off[-1, 3] == 24 and off[0, 2] == 0


def test_contracted_radial_functions_are_normalised():
    mol = M(atom="O 0 0 0; H 0 0 1.0", basis="cc-pvdz")
    for b in mol._bas:
        l, np_, nc, pe, pc = int(b[1]), int(b[2]), int(b[3]), int(b[5]), int(b[6])
        es = mol._env[pe:pe + np_]
        cs = mol._env[pc:pc + np_ * nc].reshape(nc, np_)
        ee = gaussian_int(2 * l + 2, es[:, None] + es[None, :])
        for c in range(nc):
            assert abs(cs[c] @ ee @ cs[c] - 1.0) < 1e-12


def test_cart2sph_orthonormal_harmonics():
    rng = np.random.default_rng(0)
    pts = rng.normal(size=(20000, 3))
    pts /= np.linalg.norm(pts, axis=1)[:, None]
    for l in range(2, 5):
        mono = np.stack([pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c for a, b, c in cart_components(l)], 1)
        Y = mono @ cart2sph_block(l)
        gram = Y.T @ Y * 4 * np.pi / len(pts)
        assert np.abs(gram - np.eye(2 * l + 1)).max() < 0.08   # Monte Carlo estimate
    # d(xy) coefficient: sqrt(15/(4 pi))
    assert abs(cart2sph_block(2)[1, 0] - np.sqrt(15 / (4 * np.pi))) < 1e-14


def test_decontraction_matches_ao_order():
    mol = M(atom="O 0 0 0; H 0 0 1.0", basis="cc-pvdz", cart=True)
    dc, ao_loc, orig2dc = decontract_bas(mol._bas)
    assert ao_loc[-1] == mol.nao_cart()
    ref = mol.ao_loc_nr(cart=True)
    for ish in range(mol.nbas):
        assert ao_loc[orig2dc[ish][0]] == ref[ish]
    assert (dc[:, 3] == 1).all()


def test_sparse_columns_roundtrip():
    mol = M(atom="O 0 0 0; H 0 0 1.0", basis="cc-pvdz")
    C = mol.cart2sph_coeff()
    ptr, idx, val = sparse_columns(C)
    D = np.zeros_like(C)
    for s in range(C.shape[1]):
        D[idx[ptr[s]:ptr[s + 1]], s] = val[ptr[s]:ptr[s + 1]]
    assert np.array_equal(C, D)
