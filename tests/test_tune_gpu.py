"""Autotuner on the device: the chosen launch parameters change where work
runs, not the results."""
import numpy as np
import pytest
import torch

from tests.test_oracle import checksums_close, quartet_nf

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fresh_tuner(monkeypatch):
    from ccsd_gpu_b200 import tune
    monkeypatch.delenv("CCSD_B200_TUNE_CACHE", raising=False)
    monkeypatch.setattr(tune, "_cache", None)
    monkeypatch.setattr(tune, "_have_gemm", False)
    yield
    tune.enable(False)
    tune.reset()
    for d in (0, 1):
        tune.set_heavy_nf(d, tune.ERI_HEAVY_DEFAULT[d])


def test_eri_heavy_threshold_tuning_keeps_checksums():
    from ccsd_gpu_b200 import tune, workloads
    from ccsd_gpu_b200.cuda.quartets import DeviceShells, quartet_checksums, schwarz_bounds
    sh = workloads.eri_bench_shells(4096, seed=0)
    ds = DeviceShells(sh)
    q = workloads.sample_quartets(sh, 4096, seed=5, schwarz_fn=lambda p: schwarz_bounds(ds, p))
    qd = torch.from_numpy(q).cuda()
    nf = quartet_nf(sh._bas, q)
    ref = {d: quartet_checksums(ds, qd, d).cpu().numpy() for d in (0, 1)}
    tune.enable(True)
    for d in (0, 1):
        dshare = float((sh._bas[:, 1][q].max(1) >= 2).mean())
        c = tune.tune_eri_heavy(ds, sh._bas, qd, d, dshare, sample=2048)
        assert c in tune.ERI_HEAVY_CANDIDATES[d] and tune.get_heavy_nf(d) == c
        assert tune.cache()[tune.eri_key(sh._bas, d, dshare)] == c
        for nf_cut in tune.ERI_HEAVY_CANDIDATES[d]:
            tune.set_heavy_nf(d, nf_cut)
            assert checksums_close(quartet_checksums(ds, qd, d).cpu().numpy(), ref[d], nf), (d, nf_cut)


def test_eri_path_table_and_tuning_keep_checksums():
    # every l <= 2 class forced onto each accumulation path, and the tuned
    # table, give the checksums of the compiled rule
    from ccsd_gpu_b200 import tune, workloads
    from ccsd_gpu_b200.cuda.quartets import DeviceShells, quartet_checksums, schwarz_bounds
    sh = workloads.eri_bench_shells(4096, seed=0)
    ds = DeviceShells(sh)
    q = workloads.sample_quartets(sh, 8192, seed=7, schwarz_fn=lambda p: schwarz_bounds(ds, p))
    qd = torch.from_numpy(q).cuda()
    nf = quartet_nf(sh._bas, q)
    tune.enable(True)
    for d in (0, 1):
        old = tune.get_paths(d)
        try:
            tune.set_paths(d, [0] * 81)
            ref = quartet_checksums(ds, qd, d).cpu().numpy()
            for forced in (1, 2):
                tune.set_paths(d, [forced] * 81)
                assert checksums_close(quartet_checksums(ds, qd, d).cpu().numpy(), ref, nf), (d, forced)
            tune.set_paths(d, [0] * 81)
            dshare = float((sh._bas[:, 1][q].max(1) >= 2).mean())
            t = tune.tune_eri_paths(ds, sh._bas, qd, d, dshare, per_class=1024)
            assert tune.get_paths(d) == t and set(t) <= {0, 1, 2}
            assert checksums_close(quartet_checksums(ds, qd, d).cpu().numpy(), ref, nf), (d, "tuned")
        finally:
            tune.set_paths(d, old)


def test_gemm_split_tuning_keeps_the_product():
    from ccsd_gpu_b200 import tune
    from ccsd_gpu_b200.contract import contract
    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randn(96, 8192, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(8192, 160, dtype=torch.float64, device="cuda", generator=g)
    ref = a @ b
    plain = contract("ik,kj->ij", a, b, mode="tf32x3")
    tune.enable(True)
    tuned = contract("ik,kj->ij", a, b, mode="tf32x3")
    assert "gemm:tf32x3:96:160:8192" in tune.cache()
    again = contract("ik,kj->ij", a, b, mode="tf32x3")      # held choice, no timing
    scale = float(ref.abs().max())
    for x in (plain, tuned, again):
        assert float((x - ref).abs().max()) < 1e-5 * scale
    assert torch.equal(tuned, again)


def test_gradient_with_tuning_matches_default():
    from ccsd_gpu_b200 import tune
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    mol = M(atom="O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587", basis="cc-pvdz")
    out = []
    for on in (False, True):
        tune.enable(on)
        cc = CCSD(RHF(mol).run(), precision="fp64")
        cc.kernel()
        cc.conv_tol_normt = 1e-9
        cc.solve_lambda()
        out.append(cc.nuc_grad_method().kernel())
    assert any(k.startswith("eri:1:") for k in tune.cache())
    assert any(k.startswith("eri:0:") for k in tune.cache())
    assert np.abs(out[0] - out[1]).max() < 1e-9
