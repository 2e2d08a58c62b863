"""Failure detection without a GPU fault: a bounded wait that runs out.

The tensor-core GEMM pipeline waits on mbarriers with a global-timer limit;
on expiry it records a status code and returns.  The probe kernel uses the
same wait on a barrier nothing arrives at: the host must see the code, and
the context must stay usable for the next contraction."""
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(monkeypatch):
    import ccsd_gpu_b200.contract as C
    from ccsd_gpu_b200 import _native
    monkeypatch.setattr(C, "SMALL_FLOPS", 0.0)          # the check below runs on the tensor cores
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t = time.perf_counter()
    _native.call("ccsd_b200_wait_probe", _native.ptr(st), 200_000_000, 3, _native.stream())
    torch.cuda.synchronize()
    dt = time.perf_counter() - t
    assert int(st.item()) == 3
    assert 0.15 < dt < 5.0
    # a code already present is kept (first error wins)
    _native.call("ccsd_b200_wait_probe", _native.ptr(st), 10_000_000, 7, _native.stream())
    assert int(st.item()) == 3
    # the device still works
    a = torch.randn(300, 200, dtype=torch.float64, device="cuda")
    b = torch.randn(100, 200, dtype=torch.float64, device="cuda")
    got = C.contract("mk,nk->mn", a, b)
    C.check_status()
    assert float((got - a @ b.T).abs().max() / (a @ b.T).abs().max()) < 5e-6


def test_contract_status_raises_after_expired_wait():
    """check_status() turns a recorded wait expiry into an exception and resets."""
    from ccsd_gpu_b200 import _native
    from ccsd_gpu_b200.contract import _Status, check_status
    dev = torch.device("cuda", torch.cuda.current_device())
    st = _Status.get(dev)
    _native.call("ccsd_b200_wait_probe", _native.ptr(st), 50_000_000, 2, _native.stream())
    with pytest.raises(_native.NativeError):
        check_status()
    check_status()          # reset to 0 by the raise


def test_gradient_raises_after_expired_wait(monkeypatch):
    """grad_elec_gpu must not return a gradient assembled from tensor-core
    tiles that an expired wait left unwritten: with the status already set
    the GEMMs of the gradient leave their outputs untouched and the call raises."""
    import ccsd_gpu_b200.contract as C
    from ccsd_gpu_b200 import _native
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    monkeypatch.setattr(C, "SMALL_FLOPS", 0.0)
    monkeypatch.setattr(C, "MIXED_MIN_LADDER_FLOPS", 0.0)
    mol = M(atom="O 0 0 0; H 0 -0.757 0.587; H 0 0.757 0.587", basis="sto-3g")
    cc = CCSD(RHF(mol).run(), precision="tf32x3")
    cc.kernel()
    cc.solve_lambda()
    dev = torch.device("cuda", torch.cuda.current_device())
    _native.call("ccsd_b200_wait_probe", _native.ptr(C._Status.get(dev)), 20_000_000, 5, _native.stream())
    with pytest.raises(_native.NativeError):
        cc.nuc_grad_method().kernel()
    C.check_status()            # reset by the raise
    g = cc.nuc_grad_method().kernel()
    assert np.isfinite(g).all() and np.abs(g.sum(0)).max() < 1e-8
