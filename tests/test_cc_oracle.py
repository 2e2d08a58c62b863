"""The Lambda / density-matrix oracle against golden vectors produced by the
reference's own code (tests/golden/make_cc_golden.py) -- CPU."""
import os

import numpy as np
import pytest

from oracle import cc_oracle as C
from tests.conftest import GOLDEN


# cc_small: one virtual block in the reference's loops; cc_blocked: the
# reference ran with several virtual and occupied blocks
@pytest.fixture(scope="module", params=["cc_small.npz", "cc_blocked.npz"])
def gold(request):
    return dict(np.load(os.path.join(GOLDEN, request.param)))


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_intermediates(gold):
    eris = C.mo_blocks(gold["g"], gold["t1"].shape[0])
    imds = C.make_intermediates(gold["t1"], gold["t2"], gold["fock"], eris)
    for k in ("w1", "w2", "w3", "w4", "woooo", "wvooo", "wVOov", "wvOOv", "wvvov"):
        assert rel(getattr(imds, k), gold["imds_" + k]) < 1e-12, k


def test_update_lambda_with_vvvv_ladder(gold):
    eris = C.mo_blocks(gold["g"], gold["t1"].shape[0])
    imds = C.make_intermediates(gold["t1"], gold["t2"], gold["fock"], eris)
    l1, l2 = C.update_lambda(gold["t1"], gold["t2"], gold["l1"], gold["l2"], gold["fock"], gold["mo_energy"],
                             eris, imds)
    assert rel(l1, gold["l1new"]) < 1e-12
    assert rel(l2, gold["l2new"]) < 1e-12


def test_density_matrices(gold):
    args = (gold["t1"], gold["t2"], gold["l1"], gold["l2"])
    for k, a in zip(("doo", "dov", "dvo", "dvv"), C.gamma1(*args)):
        assert rel(a, gold[k]) < 1e-12, k
    d2 = C.gamma2(*args)
    for k, a in zip(("dovov", "dvvvv", "doooo", "doovv", "dovvo", "dvvov", "dovvv", "dooov"), d2):
        if a is not None:
            assert rel(a, gold[k]) < 1e-12, k
    assert rel(C.rdm2_mo2ao_tril(d2, gold["mo_coeff"]), gold["dm2_tril"]) < 1e-12
