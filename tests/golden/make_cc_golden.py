"""Regenerate the golden Lambda / RDM fixtures by running the REFERENCE's own
Python (ccsd_gpu/gpu_ccsd_lambda.py, ccsd_gpu/gpu_ccsd_grad.py) on the CPU.

The reference imports cupy and pyscf, neither of which is installed here.  The
stand-ins below are the minimum those modules touch on the exercised paths:
  * ``cupy`` -> numpy (same function names; ``cuda.runtime.memGetInfo`` gives a
    large number so the blocking loops take one block);
  * ``pyscf.lib.prange``, ``lib.current_memory``, ``lib.logger`` (no-op timers),
    ``pyscf.cc._ccsd.make_tau`` (t2 + t1 (x) t1), ``pyscf.cc.ccsd.BLKMIN``;
  * ``mycc._add_vvvv`` = sum_cd l2[i,j,c,d] (ac|bd), the operation PySCF's
    ``_add_vvvv(None, l2, eris, with_ovvv=False, t2sym='jiba')`` performs.
Inputs: synthetic closed-shell states with 8-fold symmetric MO integrals and a
non-diagonal Fock matrix:
  * cc_small.npz    nocc=4, nvir=9, seed 0, one virtual block;
  * cc_blocked.npz  nocc=5, nvir=10, seed 1, with ``memGetInfo`` reporting
    almost no free memory, so the reference's _gpu_block_size
    (ccsd_gpu/gpu_ccsd_lambda.py:54-61) returns BLKMIN = 4 and every blocked
    loop of make_intermediates_gpu / update_lambda_gpu takes several blocks
    (virtual blocks 4+4+2, occupied blocks 4+1).
Run from the repository root:
    python tests/golden/make_cc_golden.py <reference checkout>   (or set REF_ROOT)
"""
import importlib.util
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "cc_small.npz")
OUT_BLOCKED = os.path.join(ROOT, "tests", "golden", "cc_blocked.npz")
FREE_BYTES = [1 << 40]       # what the cupy stand-in's memGetInfo reports


def _stub_modules():
    cp = types.ModuleType("cupy")
    for name in ("zeros", "einsum", "concatenate", "asarray", "diag", "dot", "zeros_like", "empty",
                 "tensordot", "tril_indices", "arange", "maximum", "minimum", "float64", "int64", "ones"):
        setattr(cp, name, getattr(np, name))
    cp.asnumpy = np.asarray
    cp.ndarray = np.ndarray
    rt = types.SimpleNamespace(memGetInfo=lambda: (FREE_BYTES[0], 1 << 40), getDeviceCount=lambda: 1)
    cp.cuda = types.SimpleNamespace(runtime=rt, Device=lambda: types.SimpleNamespace(id=0))

    pyscf = types.ModuleType("pyscf")
    lib = types.ModuleType("pyscf.lib")

    def prange(start, stop, step):
        for p0 in range(start, stop, step):
            yield p0, min(stop, p0 + step)
    lib.prange = prange
    lib.current_memory = lambda: (0.0, 0.0)
    lib.direct_sum = None
    logger = types.ModuleType("pyscf.lib.logger")

    class Logger:
        def __init__(self, *a, **k):
            pass

        def __getattr__(self, name):
            return lambda *a, **k: (0.0, 0.0)
    logger.Logger = Logger
    logger.new_logger = lambda *a, **k: Logger()
    logger.process_clock = lambda: 0.0
    logger.perf_counter = lambda: 0.0
    logger.INFO = 4
    lib.logger = logger
    lib.diis = types.SimpleNamespace(DIIS=type("DIIS", (), {}))
    cc = types.ModuleType("pyscf.cc")
    _ccsd = types.ModuleType("pyscf.cc._ccsd")
    _ccsd.make_tau = lambda t2, t1a, t1b, fac=1, out=None: t2 + np.einsum("ia,jb->ijab", t1a, t1b) * fac
    ccsd = types.ModuleType("pyscf.cc.ccsd")
    ccsd.BLKMIN = 4
    cc._ccsd, cc.ccsd = _ccsd, ccsd
    scf = types.ModuleType("pyscf.scf")
    scf.cphf = types.ModuleType("pyscf.scf.cphf")
    grad = types.ModuleType("pyscf.grad")
    grad.rhf = types.ModuleType("pyscf.grad.rhf")
    grad.mp2 = types.ModuleType("pyscf.grad.mp2")
    grad.mp2._shell_prange = grad.mp2._index_frozen_active = grad.mp2.has_frozen_orbitals = None
    pyscf.lib, pyscf.cc, pyscf.scf, pyscf.grad = lib, cc, scf, grad
    mods = {"cupy": cp, "pyscf": pyscf, "pyscf.lib": lib, "pyscf.lib.logger": logger, "pyscf.cc": cc,
            "pyscf.cc._ccsd": _ccsd, "pyscf.cc.ccsd": ccsd, "pyscf.scf": scf, "pyscf.scf.cphf": scf.cphf,
            "pyscf.grad": grad, "pyscf.grad.rhf": grad.rhf, "pyscf.grad.mp2": grad.mp2}
    sys.modules.update(mods)


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def synthetic_state(nocc=4, nvir=9, seed=0):
    rng = np.random.default_rng(seed)
    nmo = nocc + nvir
    g = rng.normal(0, 0.05, (nmo,) * 4)
    idx = np.arange(nmo)
    g *= np.exp(-0.1 * np.abs(idx[:, None] - idx[None, :]))[:, :, None, None]
    g *= np.exp(-0.1 * np.abs(idx[:, None] - idx[None, :]))[None, None]
    g = g + g.transpose(1, 0, 2, 3)
    g = g + g.transpose(0, 1, 3, 2)
    g = g + g.transpose(2, 3, 0, 1)
    g *= 0.125
    eo = np.sort(rng.uniform(-2, -0.3, nocc))
    ev = np.sort(rng.uniform(0.1, 5, nvir))
    e = np.concatenate([eo, ev])
    fock = np.diag(e) + 0.01 * (lambda a: a + a.T)(rng.normal(size=(nmo, nmo)))
    d = eo[:, None, None, None] + eo[None, :, None, None] - ev[None, None, :, None] - ev[None, None, None, :]
    t1 = rng.normal(0, 1e-2, (nocc, nvir))
    t2 = rng.normal(0, 1e-1, (nocc, nocc, nvir, nvir)) / (1 + np.abs(d))
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))
    l1 = t1 + rng.normal(0, 1e-3, t1.shape)
    l2 = t2 + rng.normal(0, 1e-3, t2.shape)
    l2 = 0.5 * (l2 + l2.transpose(1, 0, 3, 2))
    o, v = slice(0, nocc), slice(nocc, nmo)
    eris = types.SimpleNamespace(
        fock=fock, mo_energy=e, oooo=g[o, o, o, o].copy(), ovoo=g[o, v, o, o].copy(),
        ovvo=g[o, v, v, o].copy(), oovv=g[o, o, v, v].copy(), ovov=g[o, v, o, v].copy(),
        ovvv=g[o, v, v, v].copy(), vvvv=g[v, v, v, v].copy())
    eris.get_ovvv = lambda *s: eris.ovvv[s] if s else eris.ovvv
    mo_coeff = np.linalg.qr(rng.normal(size=(nmo + 2, nmo)))[0]
    return dict(g=g, fock=fock, mo_energy=e, t1=t1, t2=t2, l1=l1, l2=l2, eris=eris, mo_coeff=mo_coeff)


def ref_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT")
    if not root or not os.path.isdir(os.path.join(root, "ccsd_gpu")):
        sys.exit("usage: python %s <reference checkout>   (or set REF_ROOT)" % sys.argv[0])
    return root


def main():
    REF = ref_root()
    _stub_modules()
    lam = _load("ref_gpu_ccsd_lambda", os.path.join(REF, "ccsd_gpu", "gpu_ccsd_lambda.py"))
    grd = _load("ref_gpu_ccsd_grad", os.path.join(REF, "ccsd_gpu", "gpu_ccsd_grad.py"))
    FREE_BYTES[0] = 1 << 40
    run(lam, grd, synthetic_state(), OUT)
    FREE_BYTES[0] = 1
    run(lam, grd, synthetic_state(5, 10, seed=1), OUT_BLOCKED)


def run(lam, grd, s, path):
    eris = s["eris"]
    mycc = types.SimpleNamespace(stdout=None, verbose=0, max_memory=1e9, level_shift=0.0)
    mycc._add_vvvv = lambda t1, t2, e, with_ovvv=False, t2sym=None: np.einsum("ijcd,acbd->ijab", t2, e.vvvv)
    imds = lam.make_intermediates_gpu(mycc, s["t1"], s["t2"], eris)
    l1n, l2n = lam.update_lambda_gpu(mycc, s["t1"], s["t2"], s["l1"], s["l2"], eris, imds, use_cpu_vvvv=True)
    d1 = grd._gamma1_intermediates_gpu(mycc, s["t1"], s["t2"], s["l1"], s["l2"])
    d2 = grd._gamma2_intermediates_gpu(mycc, s["t1"], s["t2"], s["l1"], s["l2"])
    dm2 = grd._rdm2_mo2ao_gpu(mycc, d2, s["mo_coeff"])
    out = dict(g=s["g"], fock=s["fock"], mo_energy=s["mo_energy"], t1=s["t1"], t2=s["t2"], l1=s["l1"],
               l2=s["l2"], mo_coeff=s["mo_coeff"], l1new=l1n, l2new=l2n, dm2_tril=dm2)
    for k in ("w1", "w2", "w3", "w4", "woooo", "wvooo", "wVOov", "wvOOv", "wvvov"):
        out["imds_" + k] = getattr(imds, k)
    for k, v in zip(("doo", "dov", "dvo", "dvv"), d1):
        out[k] = v
    for k, v in zip(("dovov", "dvvvv", "doooo", "doovv", "dovvo", "dvvov", "dovvv", "dooov"), d2):
        if v is not None:
            out[k] = v
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
