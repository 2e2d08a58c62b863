"""Measured launch-parameter choices (autotuner), cached per shape class.

Three choices are made by timing candidates on the device:

* ERI list kernels: the Cartesian block size above which a shell quartet runs
  on the CTA-cooperative kernel instead of one warp
  (``ccsd_b200_eri_set_heavy_nf``).  Keyed by the derivative order and the
  L-class / primitive-count signature of the quartet list.
* ERI warp kernels: the accumulation path (contracted HRR or per output)
  of every L-class of a quartet list (``ccsd_b200_eri_set_paths``), kept
  only when the whole list gains.
* Split-precision GEMMs: the split-K factor, keyed by the GEMM shape
  (M, N, K) and the precision mode, i.e. by (nocc, nvir) through the shapes
  of the CCSD contractions.

The reference has fixed launch shapes (ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216,
ccsd_gpu/gpu_ccsd_lambda.py:54-61).  Choices live in a dict and, when the
environment variable ``CCSD_B200_TUNE_CACHE`` names a file, in that JSON
file, so later processes start from measured values.  Timing runs only after
``enable()``, and never while a CUDA graph is being captured (the held or
default choice is used there).
"""
import ctypes
import json
import os

import numpy as np
import torch

from . import _native

ERI_HEAVY_DEFAULT = {0: 1000, 1: 500}      # the library's compiled defaults
ERI_HEAVY_CANDIDATES = {0: (250, 500, 1000, 2000), 1: (100, 160, 250, 500, 1000)}
SPLIT_CANDIDATES = (1, 2, 4, 8, 16)

_cache = None
_gemm_tuning = False
_eri_tuning = False
_have_gemm = False


def _path():
    return os.environ.get("CCSD_B200_TUNE_CACHE") or None


def cache():
    """The choice dict {key string: value}, loaded from the cache file once."""
    global _cache, _have_gemm
    if _cache is None:
        _cache = {}
        p = _path()
        if p and os.path.exists(p):
            with open(p) as f:
                _cache.update(json.load(f))
        _have_gemm = any(k.startswith("gemm:") for k in _cache)
    return _cache


def _store(key, value):
    global _have_gemm
    cache()[key] = value
    _have_gemm = _have_gemm or key.startswith("gemm:")
    p = _path()
    if p:
        tmp = p + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache(), f, indent=1, sort_keys=True)
        os.replace(tmp, p)


def reset():
    """Forget every choice held in memory (the cache file is left alone)."""
    global _cache, _have_gemm
    _cache, _have_gemm = {}, False


def enable(on=True):
    """Tune (time candidates for) every new ERI list signature and GEMM shape
    met from now on; choices already held are used either way."""
    global _gemm_tuning, _eri_tuning
    _gemm_tuning = _eri_tuning = bool(on)


def pick(candidates, run, reps=3, timer=None):
    """(best candidate, {candidate: ms}): each candidate runs once untimed,
    then ``reps`` times between CUDA events on the current stream."""
    timer = timer or _event_ms
    times = {}
    for c in candidates:
        run(c)
        times[c] = timer(lambda: [run(c) for _ in range(reps)]) / reps
    best = min(times, key=lambda c: (times[c], candidates.index(c)))
    return best, times


def _event_ms(fn):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b)


# ---- ERI heavy-quartet threshold ------------------------------------------------
def set_heavy_nf(deriv, nf):
    rc = _native.load().ccsd_b200_eri_set_heavy_nf(int(deriv), int(nf))
    if rc != 0:
        raise _native.NativeError("ccsd_b200_eri_set_heavy_nf(%d, %d) failed" % (deriv, nf))


def get_heavy_nf(deriv):
    return int(_native.load().ccsd_b200_eri_get_heavy_nf(int(deriv)))


def eri_key(bas, deriv, dshare):
    """Signature of a quartet list: derivative order, largest l and largest
    primitive count of the shells, and the share of quartets holding a d (or
    higher) shell, rounded to a tenth."""
    bas = np.asarray(bas)
    return "eri:%d:l%d:p%d:d%.1f" % (deriv, int(bas[:, 1].max()), int(bas[:, 2].max()), dshare)


def basis_dshare(bas):
    """d-share of the list of all quartets of a basis: 1 - (share of s, p shells)^4."""
    bas = np.asarray(bas)
    return 1.0 - float((bas[:, 1] < 2).mean()) ** 4


def tune_eri_heavy(ds, bas, quartets, deriv, dshare, sample=1 << 17, candidates=None, timer=None):
    """Choose and set the heavy threshold for lists like ``quartets`` (an
    (nq, 4) int32 CUDA tensor over the shells of ``ds``: an object with
    device ``atm``, ``bas``, ``env`` and ``lmax``; ``bas`` is the host copy).

    A signature seen before (this process or the cache file) is set without
    timing.  Otherwise, when tuning is on and no graph is being captured, the
    quartet-checksum entry point is timed on an evenly spaced sample of at
    most ``sample`` quartets (L-class order kept) for each candidate; with
    tuning off the compiled default is set.  Returns the threshold in force."""
    from .cuda.quartets import quartet_checksums
    key = eri_key(bas, deriv, dshare)
    c = cache().get(key)
    if c is None:
        if not (_eri_tuning or timer) or torch.cuda.is_current_stream_capturing():
            set_heavy_nf(deriv, ERI_HEAVY_DEFAULT[deriv])
            return ERI_HEAVY_DEFAULT[deriv]
        nq = int(quartets.shape[0])
        idx = torch.unique(torch.linspace(0, nq - 1, min(sample, nq), device=quartets.device).long())
        qs = quartets[idx].contiguous()
        out = torch.empty((len(idx), 3 if deriv else 1, 2), dtype=torch.float64, device=quartets.device)

        def run(nf):
            set_heavy_nf(deriv, nf)
            quartet_checksums(ds, qs, deriv, out=out)
        c, _ = pick(list(candidates or ERI_HEAVY_CANDIDATES[deriv]), run, timer=timer)
        _store(key, int(c))
    set_heavy_nf(deriv, int(c))
    return int(c)


# ---- ERI accumulation path per L-class ----------------------------------------------
ERI_PATH_MIN = 512       # quartets of a class in the list below which the class keeps the compiled rule


def set_paths(deriv, choice):
    """Set the warp kernels' accumulation path per L-class (81 entries: 0 the
    compiled rule, 1 contracted HRR, 2 per output; class li*27+lj*9+lk*3+ll)."""
    arr = (ctypes.c_uint8 * 81)(*[int(c) for c in choice])
    rc = _native.load().ccsd_b200_eri_set_paths(int(deriv), arr, 81)
    if rc != 0:
        raise _native.NativeError("ccsd_b200_eri_set_paths failed: %s"
                                  % _native.load().ccsd_b200_last_error().decode(errors="replace"))


def get_paths(deriv):
    arr = (ctypes.c_uint8 * 81)()
    rc = _native.load().ccsd_b200_eri_get_paths(int(deriv), arr, 81)
    if rc != 0:
        raise _native.NativeError("ccsd_b200_eri_get_paths failed")
    return [int(c) for c in arr]


def class_ids(bas_dev, quartets):
    """L-class id li*27+lj*9+lk*3+ll of each quartet in its own shell order
    (-1 when a shell has l > 2), on the device."""
    l = bas_dev[:, 1].long()[quartets.long()]
    cid = l[:, 0] * 27 + l[:, 1] * 9 + l[:, 2] * 3 + l[:, 3]
    return torch.where((l <= 2).all(1), cid, torch.full_like(cid, -1))


def tune_eri_paths(ds, bas, quartets, deriv, dshare, per_class=1 << 15, timer=None):
    """Choose and set the accumulation path of every L-class of lists like
    ``quartets`` (the arguments of :func:`tune_eri_heavy`; run it first, the
    heavy threshold decides which quartets the warp kernel sees).

    For each class with at least ERI_PATH_MIN quartets whose blocks run on the
    warp kernel, the checksum entry point is timed on up to ``per_class`` of
    its quartets with the class forced onto each path, and the faster path is
    kept.  The whole table is then kept only if the (sampled) list as a whole
    runs faster with it than with the compiled rule; otherwise the compiled
    rule stays.  Returns the table in force."""
    from .cuda.quartets import quartet_checksums
    key = eri_key(bas, deriv, dshare) + ":paths"
    c = cache().get(key)
    if c is None:
        if not (_eri_tuning or timer) or torch.cuda.is_current_stream_capturing():
            set_paths(deriv, [0] * 81)
            return [0] * 81
        heavy = get_heavy_nf(deriv)
        cid = class_ids(ds.bas, quartets)
        ids, counts = torch.unique(cid, return_counts=True)
        choice = [0] * 81
        set_paths(deriv, choice)
        for k, n in zip(ids.tolist(), counts.tolist()):
            if k < 0 or n < ERI_PATH_MIN:
                continue
            ls = (k // 27, (k // 9) % 3, (k // 3) % 3, k % 3)
            if int(np.prod([(l + 1) * (l + 2) // 2 for l in ls])) > heavy:
                continue
            sel = torch.nonzero(cid == k)[:, 0]
            if len(sel) > per_class:
                sel = sel[torch.linspace(0, len(sel) - 1, per_class, device=sel.device).long()]
            qs = quartets[sel].contiguous()
            out = torch.empty((len(qs), 3 if deriv else 1, 2), dtype=torch.float64, device=quartets.device)

            def run(p, k=k, qs=qs, out=out):
                trial = list(choice)
                trial[k] = p
                set_paths(deriv, trial)
                quartet_checksums(ds, qs, deriv, out=out)
            choice[k], _ = pick([1, 2], run, timer=timer)
        # keep the table only if the list as a whole gains
        nq = int(quartets.shape[0])
        idx = torch.unique(torch.linspace(0, nq - 1, min(1 << 17, nq), device=quartets.device).long())
        qs = quartets[idx].contiguous()
        out = torch.empty((len(idx), 3 if deriv else 1, 2), dtype=torch.float64, device=quartets.device)
        tables = {0: [0] * 81, 1: choice}

        def run_all(t):
            set_paths(deriv, tables[t])
            quartet_checksums(ds, qs, deriv, out=out)
        best, _ = pick([0, 1], run_all, timer=timer)
        c = "".join(str(v) for v in tables[best])
        _store(key, c)
    set_paths(deriv, [int(v) for v in c])
    return [int(v) for v in c]


# ---- split-K factor of the split-precision GEMM ------------------------------------
def gemm_tuning_active():
    """True when a GEMM call should consult the tuner (tuning on, or choices held)."""
    if _cache is None:
        cache()
    return _gemm_tuning or _have_gemm


def gemm_split(M, N, K, mode, default, max_split, run):
    """Split-K factor for a GEMM shape.  ``run(s)`` performs the GEMM with
    split s into scratch output.  Without tuning (or while capturing) the
    held choice, else ``default``."""
    key = "gemm:%s:%d:%d:%d" % (mode, M, N, K)
    c = cache().get(key)
    if c is not None:
        return min(int(c), max_split)
    if not _gemm_tuning or torch.cuda.is_current_stream_capturing():
        return default
    cands = sorted({default} | {s for s in SPLIT_CANDIDATES if s <= max_split})
    c, _ = pick(cands, run)
    _store(key, int(c))
    return int(c)
