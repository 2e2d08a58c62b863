"""Regenerate the golden ERI fixtures from the REFERENCE's own kernels.

Needs oracle/_ref/libref_eri.so, which oracle/build_ref.py builds from the
reference checkout (fill_int2e_kernel / fill_int2e_ip1_kernel compiled for
the CPU).  Each fixture stores its own _atm/_bas/_env so the tests do not
depend on the basis tables.  Run from the repository root:

    python oracle/build_ref.py && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import eri  # noqa: E402
from ccsd_gpu_b200 import workloads  # noqa: E402
from ccsd_gpu_b200.gto import M  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")

# molecules of the reference's own ERI tests (ref: tests/test_int2e_gpu.py:20-96,
# tests/test_int2e_ip1_gpu.py:20-106), with the shell blocks stored here
MOLECULES = {
    "h2_sto3g_cart": (dict(atom="H 0 0 0; H 0 0 0.74", basis="sto-3g", cart=True), [(0, 1), (1, 2)]),
    "h2o_ccpvdz_cart": (dict(atom="O 0 0 0; H 0 0.96 0; H 0.96 0 0", basis="cc-pvdz", cart=True),
                        [(0, 1), (4, 5), (7, 8)]),
    "h2o_ccpvdz_sph": (dict(atom="O 0 0 0; H 0 0.96 0; H 0.96 0 0", basis="cc-pvdz", cart=False),
                       [(1, 2), (4, 5)]),
    "ch4_sto3g_cart": (dict(atom="C 0 0 0; H 0.629 0.629 0.629; H -0.629 -0.629 0.629; "
                                 "H -0.629 0.629 -0.629; H 0.629 -0.629 -0.629", basis="sto-3g", cart=True),
                       [(2, 3)]),
}


def main():
    assert eri.ref_available(), "build oracle/_ref first (python oracle/build_ref.py)"
    for name, (kw, blocks) in MOLECULES.items():
        mol = M(**kw)
        data = dict(atm=mol._atm, bas=mol._bas, env=mol._env, cart=np.int32(mol.cart),
                    c2s=mol.cart2sph_coeff(), blocks=np.array(blocks, dtype=np.int32))
        for b0, b1 in blocks:
            data["int2e_%d_%d" % (b0, b1)] = eri.s2kl(mol, b0, b1, 0, impl="ref")
            data["ip1_%d_%d" % (b0, b1)] = eri.s2kl(mol, b0, b1, 1, impl="ref")
        np.savez_compressed(os.path.join(OUT, "eri_%s.npz" % name), **data)
    # synthetic shells up to g (l = 4), explicit quartets, checksums
    # exponents of valence-like shells: with l = 4 and exponents near 1e4 the
    # horizontal recurrences cancel to ~1e-10 absolute in every implementation
    sh = workloads.eri_bench_shells(48, seed=7, lvals=(0, 1, 2, 3, 4), lprob=(0.2,) * 5, max_prim=3, box=3.0,
                                    exp_range=(0.1, 20.0))
    rng = np.random.default_rng(11)
    q = rng.integers(0, sh.nbas, (400, 4)).astype(np.int32)
    np.savez_compressed(os.path.join(OUT, "eri_quartets_l4.npz"), atm=sh._atm, bas=sh._bas, env=sh._env,
                        quartets=q, int2e=eri.quartet_checksums(sh, q, 0, "ref"),
                        ip1=eri.quartet_checksums(sh, q, 1, "ref"))
    for f in sorted(os.listdir(OUT)):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
