"""Split-precision tcgen05 contractions against FP64 einsum (GPU).

tf32x3 represents each FP64 operand to ~2^-24 relative; the tensor cores
accumulate in FP32 over 512-k chunks that are summed in FP64, so the error
is that of a 512-term FP32 sum on the tensor cores: up to ~4e-6 of the
largest output element (measured 3.6e-6 at K = 1000)."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("mode,tol", [("tf32x3", 5e-6), ("bf16x3", 1e-4)])
def test_plain_gemm(mode, tol):
    from ccsd_gpu_b200.contract import check_status, contract
    g = torch.Generator(device="cuda").manual_seed(0)
    for M, N, K in [(128, 128, 40), (200, 300, 100), (333, 129, 1000), (260, 140, 5000), (1, 7, 5)]:
        a = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
        b = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
        ref = a @ b.T
        got = contract("mk,nk->mn", a, b, mode=mode)
        check_status()
        assert _rel(got, ref) < tol, (M, N, K, _rel(got, ref))


def test_permuted_contraction_with_combined_operand_and_beta(monkeypatch):
    import ccsd_gpu_b200.contract as C
    from ccsd_gpu_b200.contract import check_status, contract
    monkeypatch.setattr(C, "SMALL_FLOPS", 0.0)      # keep this small case on the tensor cores
    g = torch.Generator(device="cuda").manual_seed(1)
    o, v = 6, 23
    ovvv = torch.randn(o, v, v, v, dtype=torch.float64, device="cuda", generator=g)
    t2 = torch.randn(o, o, v, v, dtype=torch.float64, device="cuda", generator=g)
    theta = [(2.0, t2), (-1.0, t2.permute(0, 1, 3, 2))]
    out = torch.randn(v, v, o, v, dtype=torch.float64, device="cuda", generator=g)
    ref = 0.5 * out - 1.5 * torch.einsum("jabd,jkcd->abkc", ovvv, 2 * t2 - t2.permute(0, 1, 3, 2))
    contract("jabd,jkcd->abkc", ovvv, theta, out=out, alpha=-1.5, beta=0.5)
    check_status()
    assert _rel(out, ref) < 5e-6


def test_outer_product_and_batch_index():
    from ccsd_gpu_b200.contract import contract
    g = torch.Generator(device="cuda").manual_seed(2)
    t1 = torch.randn(5, 9, dtype=torch.float64, device="cuda", generator=g)
    assert _rel(contract("ia,jb->ijab", t1, t1), torch.einsum("ia,jb->ijab", t1, t1)) < 5e-6
    x = torch.randn(4, 6, 7, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(4, 7, 3, dtype=torch.float64, device="cuda", generator=g)
    assert _rel(contract("bij,bjk->bik", x, y), torch.einsum("bij,bjk->bik", x, y)) < 5e-6


def test_fp64_mode_is_einsum():
    from ccsd_gpu_b200.contract import contract
    a = torch.randn(7, 8, dtype=torch.float64, device="cuda")
    b = torch.randn(9, 8, dtype=torch.float64, device="cuda")
    assert torch.allclose(contract("mk,nk->mn", a, b, mode="fp64"), a @ b.T, rtol=1e-14, atol=1e-14)


def test_tall_skinny_more_than_65535_row_tiles():
    """M = 8.4M rows (65,600 row tiles of 128): the 1-D tile raster covers it
    (the gvvvv . t1 contraction of the 2-RDM at nvir = 216 has 78,732)."""
    from ccsd_gpu_b200.contract import check_status, contract
    g = torch.Generator(device="cuda").manual_seed(3)
    M, N, K = 128 * 65600, 24, 16
    a = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
    got = contract("mk,nk->mn", a, b)
    check_status()
    assert _rel(got, a @ b.T) < 5e-6


def test_packed_operand_cache_follows_in_place_updates():
    from ccsd_gpu_b200.contract import _pack_cache, check_status, contract, mark_constant
    g = torch.Generator(device="cuda").manual_seed(4)
    a = torch.randn(600, 800, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(400, 800, dtype=torch.float64, device="cuda", generator=g)
    mark_constant(b)
    n0 = len(_pack_cache)
    r1 = contract("mk,nk->mn", a, b)
    assert len(_pack_cache) == n0 + 1
    r2 = contract("mk,nk->mn", a, b)
    assert torch.equal(r1, r2)
    b.mul_(2.0)                       # bumps the version counter: the packed copy is stale
    r3 = contract("mk,nk->mn", a, b)
    check_status()
    assert _rel(r3, a @ b.T) < 5e-6
    del b
    assert len(_pack_cache) <= n0 + 1


def test_split_k_skinny_output_long_k():
    """Output of 2 x 1 tiles with K = 300,000: the k blocks are split over
    CTAs (partials summed in a fixed order by a second kernel); beta applied once."""
    from ccsd_gpu_b200.contract import STATS, check_status, contract
    g = torch.Generator(device="cuda").manual_seed(5)
    M, N, K = 256, 64, 300000
    a = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
    out = torch.randn(M, N, dtype=torch.float64, device="cuda", generator=g)
    ref = 0.25 * out + 2.0 * (a @ b.T)
    n0 = STATS["launches"]
    contract("mk,nk->mn", a, b, out=out, alpha=2.0, beta=0.25)
    check_status()
    assert STATS["launches"] - n0 == 4          # two packs, GEMM, split-K reduction
    assert _rel(out, ref) < 5e-6
    again = contract("mk,nk->mn", a, b)
    assert torch.equal(again, contract("mk,nk->mn", a, b))   # fixed summation order


def test_memory_bound_shapes_take_the_fp64_route():
    """K <= 32 or fewer than 12 flop per byte: FP64 cuBLAS, no native launch."""
    from ccsd_gpu_b200.contract import STATS, contract
    g = torch.Generator(device="cuda").manual_seed(6)
    w = torch.randn(24, 24, dtype=torch.float64, device="cuda", generator=g)
    l2 = torch.randn(24, 24, 30, 30, dtype=torch.float64, device="cuda", generator=g)
    n0 = STATS["launches"]
    got = contract("jk,kiba->jiba", w, l2)
    assert STATS["launches"] == n0
    assert torch.allclose(got, torch.einsum("jk,kiba->jiba", w, l2), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("mode,tol", [("tf32x3", 5e-6), ("bf16x3", 1e-4)])
def test_tensor_route_on_tiny_and_ragged_shapes(mode, tol, monkeypatch):
    """The tcgen05 route itself on shapes the dispatcher would send to FP64:
    one row, K below one TMA box, rows past the operand read as zeros."""
    import ccsd_gpu_b200.contract as C
    monkeypatch.setattr(C, "LOW_INTENSITY_K", 0)
    monkeypatch.setattr(C, "LOW_INTENSITY_FLOP_PER_BYTE", 0.0)
    monkeypatch.setattr(C, "SMALL_FLOPS", 0.0)
    g = torch.Generator(device="cuda").manual_seed(7)
    for M, N, K in [(1, 7, 5), (128, 128, 40), (24, 5000, 24), (3, 1, 1)]:
        a = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
        b = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
        n0 = C.STATS["launches"]
        got = C.contract("mk,nk->mn", a, b, mode=mode)
        C.check_status()
        assert C.STATS["launches"] - n0 >= 3
        assert _rel(got, a @ b.T) < tol, (M, N, K)


@pytest.mark.parametrize("mode,tol", [("tf32x3", 5e-6), ("bf16x3", 1e-4)])
def test_transposing_gather_pack(mode, tol, monkeypatch):
    """Operands stored contiguous along the packed rows (here A as (K, M) and
    B as (K, N)) take the shared-memory transposing pack; ragged tile edges."""
    import ccsd_gpu_b200.contract as C
    monkeypatch.setattr(C, "SMALL_FLOPS", 0.0)
    g = torch.Generator(device="cuda").manual_seed(8)
    for M, N, K in [(333, 200, 129), (64, 1000, 300), (5, 7, 40)]:
        a = torch.randn(K, M, dtype=torch.float64, device="cuda", generator=g)
        b = torch.randn(K, N, dtype=torch.float64, device="cuda", generator=g)
        got = C.contract("km,kn->mn", a, b, mode=mode)
        C.check_status()
        assert _rel(got, a.T @ b) < tol, (M, N, K)
