"""The oracle against the reference's golden vectors and against mathematics (CPU)."""
import os
import re

import numpy as np
import pytest

from oracle import eri
from tests.conftest import GOLDEN, ROOT

RTOL = 1e-10


def block_close(a, b, rtol=RTOL, atol=1e-12):
    scale = np.abs(b).max()
    return np.abs(a - b).max() <= rtol * scale + atol


def test_rys_moment_identity():
    """sum_i w_i u_i^k = F_k(x), k < 2n (cf. ref: ccsd_gpu/cuda/int2e_ip1_module.py:212-220)."""
    for n in range(1, 10):
        for x in [0.0, 1e-9, 1e-4, 0.7, 3.3, 12.0, 38.0, 39.9 + 5 * n, 40.1 + 5 * n, 250.0, 1e5]:
            u, w = eri.rys_roots(n, x)
            F = eri.boys(2 * n - 1, x)
            assert np.all(np.diff(u) > 0) and np.all(u > 0) and np.all(u < 1)
            for k in range(2 * n):
                assert abs((w * u ** k).sum() - F[k]) <= 2e-14 * F[k], (n, x, k)


def _load_tables():
    txt = open(os.path.join(ROOT, "ccsd_gpu_b200", "csrc", "rys_tables.inc")).read()

    def arr(name):
        m = re.search(r"%s\[\d+\] = \{(.*?)\};" % name, txt, re.S)
        return np.array([float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()])
    return arr("RYS_CHEB_OFFSET").astype(int), arr("RYS_CHEB"), arr("RYS_LARGEX_U"), arr("RYS_LARGEX_W")


def table_roots(tables, n, x):
    off, cheb, lu, lw = tables
    if x < 40 + 5 * n:
        it = min(int(x / 2.5), 16 + 2 * n - 1)
        t = (x - it * 2.5) * 0.8 - 1
        base = off[n - 1] + it * 2 * n * 14
        v = [np.polynomial.chebyshev.chebval(t, cheb[base + s * 14: base + (s + 1) * 14]) for s in range(2 * n)]
        return np.array(v[:n]), np.array(v[n:])
    o = n * (n - 1) // 2
    return lu[o:o + n] / x, lw[o:o + n] / np.sqrt(x)


def test_device_rys_tables_match_oracle():
    """The kernels' Chebyshev tables (evaluated here on the host) vs the oracle's roots."""
    tables = _load_tables()
    rng = np.random.default_rng(3)
    for n in range(1, 10):
        xs = np.concatenate([[0.0, 1e-12, 2.5, 39.99 + 5 * n, 40.01 + 5 * n, 1e3],
                             rng.uniform(0, 45 + 5 * n, 40)])
        for x in xs:
            u, w = table_roots(tables, n, x)
            uo, wo = eri.rys_roots(n, x)
            assert np.abs(u - uo).max() <= 1e-13 * uo.max(), (n, x)
            assert np.abs(w - wo).max() <= 1e-13 * wo.max(), (n, x)


def test_reference_rys_agrees_with_oracle():
    if not eri.ref_available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    for n in range(1, 10):
        for x in [1e-3, 0.5, 4.0, 17.0, 33.0, 120.0]:
            ur, wr = eri.ref_rys_roots(n, x)
            o = np.argsort(ur)
            u, w = eri.rys_roots(n, x)
            assert np.abs(u - ur[o]).max() <= 1e-11 * u.max()
            assert np.abs(w - wr[o]).max() <= 1e-11 * w.max()


def test_oracle_matches_reference_golden(golden_mols):
    for name, (mol, d) in golden_mols.items():
        for b0, b1 in d["blocks"]:
            got0 = eri.s2kl(mol, int(b0), int(b1), 0)
            got1 = eri.s2kl(mol, int(b0), int(b1), 1)
            assert block_close(got0, d["int2e_%d_%d" % (b0, b1)]), (name, b0, b1)
            assert block_close(got1, d["ip1_%d_%d" % (b0, b1)]), (name, b0, b1)


def checksums_close(a, b, nf, rtol=RTOL, atol=1e-12):
    """Checksums of two integral sets agree as if every element obeyed
    |dv| <= rtol |v| + atol (the reference's own ERI tests use atol = 1e-10,
    ref: tests/test_int2e_gpu.py:99-163)."""
    nf = np.asarray(nf, dtype=np.float64)[:, None]
    s2 = np.abs(b[..., 1])
    bound = 2 * np.sqrt(nf * s2)
    ok1 = np.abs(a[..., 0] - b[..., 0]) <= rtol * bound + 2 * atol * nf
    ok2 = np.abs(a[..., 1] - b[..., 1]) <= 2 * rtol * s2 + 2 * atol * np.sqrt(nf * s2) + nf * atol ** 2
    return bool(ok1.all() and ok2.all())


def quartet_nf(bas, q):
    l = bas[:, 1][q]
    return np.prod((l + 1) * (l + 2) // 2, axis=1)


def test_oracle_quartets_up_to_g_match_reference_golden():
    d = dict(np.load(os.path.join(GOLDEN, "eri_quartets_l4.npz")))
    from ccsd_gpu_b200.workloads import ShellSet
    sh = ShellSet(d["atm"], d["bas"], d["env"])
    nf = quartet_nf(d["bas"], d["quartets"])
    assert checksums_close(eri.quartet_checksums(sh, d["quartets"], 0), d["int2e"], nf)
    assert checksums_close(eri.quartet_checksums(sh, d["quartets"], 1), d["ip1"], nf)
