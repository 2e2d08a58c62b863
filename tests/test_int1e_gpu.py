"""One-electron integral kernel (ccsd_b200_int1e_cart) against the
McMurchie-Davidson oracle, every operator, with d shells.

These replace libcint's int1e_* that the reference reaches through PySCF's
hcore_generator and get_ovlp (ref: ccsd_gpu/gpu_ccsd_grad.py:554-584); the
derivative operators (ip*) and the 1/r_C operator around each nucleus
(iprinv) carry the one-electron part of the gradient."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPS = ["int1e_ovlp", "int1e_kin", "int1e_nuc", "int1e_rinv", "int1e_ipovlp", "int1e_ipkin", "int1e_ipnuc",
       "int1e_iprinv"]


@pytest.fixture(scope="module", params=[True, False], ids=["cart", "sph"])
def mol(request):
    from ccsd_gpu_b200.gto import M
    # cc-pVDZ oxygen carries a d shell; the geometry has no symmetry
    return M(atom="O 0 0 0; H 0 0.757 0.587; H 0.1 -0.757 0.587", basis="cc-pvdz", cart=request.param)


@pytest.mark.parametrize("name", OPS)
def test_int1e_matches_oracle(mol, name):
    from ccsd_gpu_b200.int1e import intor1e
    from oracle import int1e_oracle as O
    origins = range(mol.natm) if "rinv" in name else [None]
    for a in origins:
        got = intor1e(mol, name, origin_atom=a).cpu().numpy()
        ref = O.int1e(mol, name, origin_atom=a)
        assert got.shape == ref.shape
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max() + 1e-14, (name, a)


def test_int1e_derivative_translational_invariance(mol):
    """sum over both centres of d/dR <i|O|j> vanishes for the overlap and
    kinetic operators: <d_i i|j> + <i|d_j j> = 0, i.e. ip + ip^T = 0."""
    from ccsd_gpu_b200.int1e import intor1e
    for name in ("int1e_ipovlp", "int1e_ipkin"):
        g = intor1e(mol, name).cpu().numpy()
        assert np.abs(g + g.transpose(0, 2, 1)).max() < 1e-12, name
