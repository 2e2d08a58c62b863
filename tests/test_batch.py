"""Shape-batched solves of many molecules (ccsd_gpu_b200.batch).

CPU: the batched DIIS and the vmap-batched T / Lambda update bodies equal
their per-molecule counterparts.  GPU: batched gradients of a set of small
molecules of two shapes equal the molecule-by-molecule chain."""
import os
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from tests.conftest import GOLDEN


def test_batched_diis_matches_per_molecule_diis():
    from ccsd_gpu_b200.batch import _BatchDIIS
    from ccsd_gpu_b200.gpu_ccsd_lambda import DIIS
    g = torch.Generator().manual_seed(0)
    B, n = 3, 40
    bd = _BatchDIIS(B, n, 5, torch.device("cpu"))
    singles = [DIIS(5) for _ in range(B)]
    x = torch.randn(B, n, generator=g, dtype=torch.float64)
    for it in range(9):
        e = 0.5 ** it * torch.randn(B, n, generator=g, dtype=torch.float64)
        got = bd.update(x + e, e)
        ref = torch.stack([d.update(x[b] + e[b], e[b]) for b, d in enumerate(singles)])
        assert float((got - ref).abs().max()) < 1e-10
        x = got


def test_vmap_update_bodies_match_per_molecule(monkeypatch):
    """The batched T and Lambda bodies (one vmap over the group) give each
    molecule's own update, on three perturbed copies of a golden state."""
    import ccsd_gpu_b200._native as N
    import ccsd_gpu_b200.batch as Bt
    import ccsd_gpu_b200.gpu_ccsd_lambda as GL
    from oracle import cc_oracle as C
    monkeypatch.setattr(N, "require_cuda", lambda *a, **k: None)     # FP64 bodies are plain torch ops
    monkeypatch.setattr(GL, "_dev", lambda: torch.device("cpu"))
    d = dict(np.load(os.path.join(GOLDEN, "cc_small.npz")))
    e = C.mo_blocks(d["g"], d["t1"].shape[0])
    B = 3
    tt = lambda x: torch.as_tensor(np.ascontiguousarray(x))     # noqa: E731
    consts = {k: torch.stack([tt(getattr(e, k)) * (1 + 0.01 * b) for b in range(B)])
              for k in ("oooo", "ovoo", "ovvo", "oovv", "ovov", "ovvv", "vvvv")}
    consts["fock"] = torch.stack([tt(d["fock"])] * B)
    consts["mo_energy"] = torch.stack([tt(d["mo_energy"])] * B)
    t1 = torch.stack([tt(d["t1"]) * (1 + 0.1 * b) for b in range(B)])
    t2 = torch.stack([tt(d["t2"])] * B)
    got_t = torch.func.vmap(Bt._t_body)(consts, t1, t2)
    lc = dict(consts, t1=t1, t2=t2)
    imds = torch.func.vmap(Bt._imds_body)(lc)
    lc.update({"i_" + k: v for k, v in zip(Bt._IMDS, imds)})
    got_l = torch.func.vmap(Bt._l_body)(lc, t1, t2)
    for b in range(B):
        cb = {k: v[b] for k, v in lc.items()}
        ref_t = Bt._t_body(cb, t1[b], t2[b])
        ref_l = Bt._l_body(cb, t1[b], t2[b])
        for got, ref in ((got_t, ref_t), (got_l, ref_l)):
            assert float((got[0][b] - ref[0]).abs().max()) < 1e-14
            assert float((got[1][b] - ref[1]).abs().max()) < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["fp64", "tf32x3"])
def test_batched_gradients_match_serial(mode):
    from ccsd_gpu_b200 import batch, workloads
    from ccsd_gpu_b200.gto import M
    rng = np.random.default_rng(3)
    mols = []
    for n in (1, 2, 1, 2, 1):
        s, x = workloads.water_cluster_atoms(n, rng)
        mols.append(M(atom=workloads.atom_string(s, x), basis="cc-pvdz"))
    got = batch.gradients(mols, mode, batched=True)
    ref = batch.gradients(mols, mode, batched=False)
    for g, r in zip(got, ref):
        assert g.shape == r.shape
        assert np.abs(g - r).max() < 1e-8
        assert np.abs(g.sum(0)).max() < 1e-8
