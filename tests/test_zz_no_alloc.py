"""The allocation-free spherical transform, for callers that cannot allocate.

Some callers of this library cannot call cudaMalloc (a host application that
manages the device through its own pool, or one that forbids allocation while
a step runs).  ccsd_b200_cart2sph_s2kl_noalloc keeps the transform's
intermediate in a built-in device array instead of a caller buffer.  These
tests call it through the C ABI and compare it with ccsd_b200_cart2sph_s2kl,
which takes caller scratch, on two calls in a row with different block sizes,
so a stale intermediate from the first call would show up in the second.
They also check that a block too large for the built-in array is refused.
The file is named to be collected last.
"""
import numpy as np
import pytest
import torch

from tests.test_oracle import block_close

pytestmark = pytest.mark.gpu


def _cart_block(mol, b0, b1, deriv):
    """Cartesian s2kl block from the ERI entry point, plus what the transform needs."""
    from ccsd_gpu_b200 import _native
    from ccsd_gpu_b200.cuda._eri import heavy_quartets
    from ccsd_gpu_b200.cuda.basis import get_basis_cached, upload_geometry
    dev = torch.device("cuda", torch.cuda.current_device())
    topo = get_basis_cached(mol, dev)
    atm, env = upload_geometry(mol, dev)
    d0, d1 = topo.orig2dc[b0][0], topo.orig2dc[b1 - 1][-1] + 1
    nfc = int(topo.dc_ao_loc[d1] - topo.dc_ao_loc[d0])
    naoc = topo.nao_cart
    ncomp = 3 if deriv else 1
    cart = torch.empty((ncomp, nfc, naoc, naoc * (naoc + 1) // 2), dtype=torch.float64, device=dev)
    hq = heavy_quartets(topo, d0, d1, deriv)
    _native.call("ccsd_b200_eri_s2kl_cart", deriv, _native.ptr(atm), _native.ptr(topo.bas_dev), _native.ptr(env),
                 topo.dc_nbas, _native.ptr(topo.ao_loc_dev), d0, d1, naoc, topo.lmax, _native.ptr(hq),
                 int(hq.shape[0]), _native.ptr(cart), _native.stream())
    sph = topo.sph()
    ls = sph["ao_loc_sph"]
    return cart, topo, sph, int(ls[b1] - ls[b0]), int(ls[-1])


def _both(mol, b0, b1, deriv):
    from ccsd_gpu_b200 import _native
    cart, topo, sph, nfs, naos = _cart_block(mol, b0, b1, deriv)
    ncomp, nfc, naoc = cart.shape[0], cart.shape[1], cart.shape[2]
    npc, nps = naoc * (naoc + 1) // 2, naos * (naos + 1) // 2
    pi, ii, vi = topo.sph_block(b0, b1)
    common = (_native.ptr(pi), _native.ptr(ii), _native.ptr(vi), _native.ptr(sph["ptr"]), _native.ptr(sph["idx"]),
              _native.ptr(sph["val"]), _native.stream())
    tmp = torch.empty((ncomp, nfs, naos, npc), dtype=torch.float64, device=cart.device)
    ref = torch.empty((ncomp, nfs, naos, nps), dtype=torch.float64, device=cart.device)
    _native.call("ccsd_b200_cart2sph_s2kl", _native.ptr(cart), _native.ptr(tmp), _native.ptr(ref), ncomp, nfc, naoc,
                 nfs, naos, *common)
    got = torch.full_like(ref, float("nan"))
    _native.call("ccsd_b200_cart2sph_s2kl_noalloc", _native.ptr(cart), _native.ptr(got), ncomp, nfc, naoc, nfs,
                 naos, *common)
    torch.cuda.synchronize()
    return got.cpu().numpy(), ref.cpu().numpy()


def test_no_alloc_transform_matches_scratch_variant_twice():
    from ccsd_gpu_b200.gto import M
    mol = M(atom="O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587", basis="cc-pvdz", cart=False)
    for b0, b1, deriv in [(0, mol.nbas, 1), (4, 5, 0)]:
        got, ref = _both(mol, b0, b1, deriv)
        assert np.isfinite(got).all()
        assert block_close(got, ref), (b0, b1, deriv)


def test_no_alloc_transform_refuses_blocks_beyond_its_buffer():
    from ccsd_gpu_b200 import _native
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    i = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = _native.ptr
    with pytest.raises(_native.NativeError, match="32 MiB"):
        # 3 x 500 x 500 rows x 125250 pairs: far beyond the built-in buffer; refused before any launch
        _native.call("ccsd_b200_cart2sph_s2kl_noalloc", p(x), p(x), 3, 10, 500, 500, 500, p(i), p(i), p(x), p(i),
                     p(i), p(x), _native.stream())
