"""ctypes binding of ``libccsdb200.so`` (the extern "C" API of include/ccsd_b200.h).

There is no CPU path behind these functions: if the library is missing or a
CUDA device is not available the call raises.
"""
import collections
import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libccsdb200.so")

_c_int = ctypes.c_int
_c_ll = ctypes.c_longlong
_c_dbl = ctypes.c_double
_vp = ctypes.c_void_p

# name -> (restype, argtypes); must match include/ccsd_b200.h
SIGNATURES = {
    "ccsd_b200_last_error": (ctypes.c_char_p, []),
    "ccsd_b200_eri_s2kl_cart": (_c_int, [_c_int, _vp, _vp, _vp, _c_int, _vp, _c_int, _c_int, _c_int,
                                         _c_int, _vp, _c_ll, _vp, _vp]),
    "ccsd_b200_eri_s2kl_sph": (_c_int, [_c_int, _vp, _vp, _vp, _c_int, _vp, _vp, _vp, _c_int, _c_int, _c_int,
                                        _c_int, _vp, _c_ll, _vp, _vp]),
    "ccsd_b200_eri_quartet_checksums": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _c_ll, _c_int, _vp, _vp]),
    "ccsd_b200_eri_set_heavy_nf": (_c_int, [_c_int, _c_int]),
    "ccsd_b200_eri_get_heavy_nf": (_c_int, [_c_int]),
    "ccsd_b200_eri_set_paths": (_c_int, [_c_int, _vp, _c_int]),
    "ccsd_b200_eri_get_paths": (_c_int, [_c_int, _vp, _c_int]),
    "ccsd_b200_cart2sph_s2kl": (_c_int, [_vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int,
                                         _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ccsd_b200_fp64_fma_probe": (_c_int, [_vp, _c_int, _c_int, _vp]),
    "ccsd_b200_int1e_cart": (_c_int, [_c_int, _vp, _c_int, _vp, _c_int, _vp, _vp, _c_int, _c_int, _vp, _vp]),
    "ccsd_b200_cart2sph_s2kl_noalloc": (_c_int, [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int,
                                                 _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ccsd_b200_split_pack": (_c_int, [_c_int, _vp, _vp, _vp, _c_dbl, _vp, _vp, _vp, _c_dbl, _c_int, _c_int,
                                      _c_int, _c_int, _vp, _vp, _c_int, _vp]),
    "ccsd_b200_eri_full_cart": (_c_int, [_vp, _vp, _vp, _vp, _c_int, _vp, _c_ll, _c_int, _vp, _vp]),
    "ccsd_b200_eri_ip1_contract": (_c_int, [_vp, _vp, _vp, _vp, _c_int, _vp, _vp, _c_ll, _vp, _c_int, _c_int, _vp,
                                            _vp, _vp]),
    "ccsd_b200_eri_ip1_contract_rows": (_c_int, [_vp, _vp, _vp, _vp, _c_int, _vp, _c_int, _c_int, _vp, _c_ll, _vp,
                                                 _c_int, _c_int, _vp, _vp, _vp]),
    "ccsd_b200_wait_probe": (_c_int, [_vp, _c_ll, _c_int, _vp]),
    "ccsd_b200_tc_split_gemm": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int,
                                         _vp, _vp, _vp, _c_dbl, _c_dbl, _c_int, _vp, _vp, _vp]),
}


class NativeError(RuntimeError):
    """Error status returned by a libccsdb200 entry point."""


_lib = None


def load():
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("%s is missing: build it with `python -m ccsd_gpu_b200.build`" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


# entry-point calls made through call() (each enqueues at least one kernel),
# read by the benchmarks
CALLS = collections.Counter()


def call(name, *args):
    CALLS[name] += 1
    rc = getattr(load(), name)(*args)
    if rc != 0:
        raise NativeError("%s failed (status %d): %s"
                          % (name, rc, load().ccsd_b200_last_error().decode(errors="replace")))
    return rc


def require_cuda(t=None):
    if not torch.cuda.is_available():
        raise RuntimeError("ccsd_gpu_b200 needs a CUDA device; there is no CPU fallback")
    if t is not None and not t.is_cuda:
        raise ValueError("expected a CUDA tensor")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def stream(s=None):
    s = s if s is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
