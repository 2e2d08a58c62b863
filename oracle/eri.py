"""ORACLE -- test infrastructure only.

ctypes front end for
  * liboracle_eri.so : the C restatement in eri_oracle.c (always available,
    built by ``build()`` from this directory with gcc);
  * _ref/libref_eri.so : the reference's own kernels compiled for the CPU by
    build_ref.py (available where the reference checkout was present when
    the tree was built).
Both produce the s2kl integral block of compute_int2e_gpu /
compute_int2e_ip1_gpu (ref: ccsd_gpu/cuda/int2e_gpu.py:186-215,
ccsd_gpu/cuda/int2e_ip1_gpu.py:296-326) on the CPU.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_eri.so")
REF_SO = os.path.join(HERE, "_ref", "libref_eri.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")


def build_oracle():
    src = os.path.join(HERE, "eri_oracle.c")
    if os.path.exists(ORACLE_SO) and os.path.getmtime(ORACLE_SO) >= os.path.getmtime(src):
        return ORACLE_SO
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11",
                           src, "-o", ORACLE_SO, "-lm"])
    return ORACLE_SO


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.oracle_rys_roots.argtypes = [ctypes.c_int, ctypes.c_double, _f64p, _f64p]
        _lib.oracle_boys.argtypes = [ctypes.c_int, ctypes.c_double, _f64p]
        _lib.oracle_eri_s2kl.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, _f64p,
                                         _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
        _lib.oracle_eri_quartet.argtypes = [_i32p, _i32p, _f64p] + [ctypes.c_int] * 5 + [_f64p]
        _lib.oracle_eri_quartet_checksums.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _i32p,
                                                      ctypes.c_long, _f64p]
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
        _ref.ref_eri_cart.argtypes = [ctypes.c_int, _f64p, _i32p, _i32p, _f64p, _i32p,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      _i32p, ctypes.c_int]
        _ref.ref_rys_roots.argtypes = [ctypes.c_int, ctypes.c_double, _f64p, _f64p]
        _ref.ref_eri_quartet_checksums.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _i32p,
                                                   ctypes.c_long, _f64p]
    return _ref


def rys_roots(n, x):
    u = np.zeros(n)
    w = np.zeros(n)
    lib().oracle_rys_roots(n, float(x), u, w)
    return u, w


def ref_rys_roots(n, x):
    u = np.zeros(n)
    w = np.zeros(n)
    ref().ref_rys_roots(n, float(x), u, w)
    return u, w


def boys(mmax, x):
    F = np.zeros(mmax + 1)
    lib().oracle_boys(mmax, float(x), F)
    return F


def _arrays(mol):
    return (np.ascontiguousarray(mol._atm, dtype=np.int32),
            np.ascontiguousarray(mol._bas, dtype=np.int32),
            np.ascontiguousarray(mol._env, dtype=np.float64))


def cart_s2kl(mol, b0, b1, deriv=0):
    """Cartesian s2kl block from the C restatement: (ncomp, nf, nao, nao_pair)."""
    atm, bas, env = _arrays(mol)
    ao_loc = np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int32)
    nao = int(ao_loc[-1])
    nf = int(ao_loc[b1] - ao_loc[b0])
    ncomp = 3 if deriv else 1
    out = np.zeros(ncomp * nf * nao * (nao * (nao + 1) // 2))
    lib().oracle_eri_s2kl(atm, len(atm), bas, len(bas), env, ao_loc, b0, b1, int(deriv), out)
    return out.reshape(ncomp, nf, nao, -1)


def _decontract(bas):
    rows, orig2dc = [], []
    for ish in range(len(bas)):
        nctr, nprim, pc = int(bas[ish, 3]), int(bas[ish, 2]), int(bas[ish, 6])
        idx = []
        for c in range(nctr):
            r = bas[ish].copy()
            r[3] = 1
            r[6] = pc + c * nprim
            idx.append(len(rows))
            rows.append(r)
        orig2dc.append(idx)
    dc = np.ascontiguousarray(np.array(rows, dtype=np.int32))
    l = dc[:, 1]
    ao_loc = np.zeros(len(dc) + 1, dtype=np.int32)
    np.cumsum((l + 1) * (l + 2) // 2, out=ao_loc[1:])
    return dc, ao_loc, orig2dc


def ref_cart_s2kl(mol, b0, b1, deriv=0):
    """Cartesian s2kl block from the reference kernels run on the CPU."""
    atm, bas, env = _arrays(mol)
    dc, ao_loc, orig2dc = _decontract(bas)
    nbas = len(dc)
    nao = int(ao_loc[-1])
    k, l = np.tril_indices(nbas)
    pairs = np.ascontiguousarray(np.stack([k, l], 1).ravel().astype(np.int32))
    d0, d1 = orig2dc[b0][0], orig2dc[b1 - 1][-1] + 1
    nf = int(ao_loc[d1] - ao_loc[d0])
    ncomp = 3 if deriv else 1
    out = np.zeros(ncomp * nf * nao * (nao * (nao + 1) // 2))
    ref().ref_eri_cart(int(deriv), out, atm, dc, env, ao_loc, d0, d1, nbas, nao,
                       pairs, len(pairs) // 2)
    return out.reshape(ncomp, nf, nao, -1)


def cart_to_sph(block, mol, b0, b1):
    """(ncomp, nf_cart, nao_cart, npair_cart) -> spherical, for any mol."""
    C = mol.cart2sph_coeff()
    lc = mol.ao_loc_nr(cart=True)
    ls = mol.ao_loc_nr(cart=False)
    Ci = C[lc[b0]:lc[b1], ls[b0]:ls[b1]]
    ncomp, nf, nc, _ = block.shape
    ns = C.shape[1]
    k, l = np.tril_indices(nc)
    full = np.zeros((ncomp, nf, nc, nc, nc))
    full[..., k, l] = block
    full[..., l, k] = block
    out = np.einsum("xijkl,ia,jb,kc,ld->xabcd", full, Ci, C, C, C, optimize=True)
    ks, ls_ = np.tril_indices(ns)
    return out[..., ks, ls_]


def s2kl(mol, b0, b1, deriv=0, impl="oracle"):
    """Block in the molecule's native basis (Cartesian or spherical)."""
    fn = cart_s2kl if impl == "oracle" else ref_cart_s2kl
    cart = fn(mol, b0, b1, deriv)
    if not mol.cart:
        cart = cart_to_sph(cart, mol, b0, b1)
    return cart if deriv else cart[0]


def quartet_checksums(shells, quartets, deriv, impl="oracle"):
    """(nq, ncomp, 2) checksums of explicit quartets on the CPU (all OpenMP threads)."""
    atm, bas, env = _arrays(shells)
    q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
    ncomp = 3 if deriv else 1
    out = np.zeros(len(q) * ncomp * 2)
    fn = lib().oracle_eri_quartet_checksums if impl == "oracle" else ref().ref_eri_quartet_checksums
    fn(int(deriv), atm, bas, env, q.ravel(), len(q), out)
    return out.reshape(len(q), ncomp, 2)
