"""Tensor contractions for the Lambda / density-matrix path.

``contract(spec, a, b, out=..., alpha=1, beta=0, mode=...)`` evaluates one
two-operand einsum ``spec`` (e.g. ``"jabd,jkcd->abkc"``) as a GEMM
D[m, n] = sum_k A[m, k] B[n, k]:

  * M = indices of ``a`` that survive, N = indices of ``b`` that survive, K = the
    summed indices; M and N are ordered as in the output string.  An index
    present in all three is a batch index and is looped on the host.
  * mode "tf32x3" / "bf16x3": the operands are gathered through element-offset
    tables, split into hi + lo parts and packed for TMA by one kernel
    (``ccsd_b200_split_pack``), multiplied on the tcgen05 tensor cores
    (``ccsd_b200_tc_split_gemm``: hi*hi + hi*lo + lo*hi, FP32 accumulation in
    512-k chunks drained to FP64), and the result is scattered straight into
    ``out`` with alpha/beta -- no permuted copy of any operand or of the result
    is materialised.  An operand may be a linear combination of two views
    (``[(2.0, t2), (-1.0, t2p)]``), which fuses the ``2 t - t^T`` patterns of
    the CCSD equations into the pack.
  * mode "fp64": ``torch.einsum`` in float64 (cuBLAS DGEMM): the plain FP64 GPU
    path the split-precision modes are measured against.
"""
import weakref

import numpy as np
import torch

from . import _native, tune

KIND = {"tf32x3": 0, "bf16x3": 1}
MODES = ("fp64", "tf32x3", "bf16x3")
_BM = 128
_KALIGN = {"tf32x3": 4, "bf16x3": 8}      # packed rows start on 16-byte boundaries
_KSTEP = {"tf32x3": 32, "bf16x3": 64}     # k per 128-byte TMA box row


def _parse(spec):
    lhs, out = spec.replace(" ", "").split("->")
    a, b = lhs.split(",")
    return a, b, out


def _terms(x):
    if isinstance(x, torch.Tensor):
        return [(1.0, x)]
    return [(float(c), t) for c, t in x]


def _offsets(idx_order, sub, shape_map, tensor):
    """Element offsets over the row-major grid of idx_order for a tensor indexed by `sub`."""
    if not idx_order:
        return np.zeros(1, dtype=np.int64)
    st = dict(zip(sub, tensor.stride()))
    off = np.zeros(1, dtype=np.int64)
    for ix in idx_order:
        n = shape_map[ix]
        off = (off[:, None] + np.arange(n, dtype=np.int64)[None, :] * st.get(ix, 0)).ravel()
    return off


class _Status:
    buf = {}

    @classmethod
    def get(cls, dev):
        t = cls.buf.get(dev)
        if t is None:
            t = torch.zeros(1, dtype=torch.int32, device=dev)
            cls.buf[dev] = t
        return t


def check_status(device=None):
    """Raise if any tensor-core GEMM since the last check recorded an expired wait."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    st = _Status.get(dev)
    v = int(st.item())
    if v:
        st.zero_()
        raise _native.NativeError("tensor-core GEMM pipeline wait expired (code %d)" % v)


_off_cache = {}

# running totals, read by benchmarks: algorithmic FLOPs (2 M N K per GEMM, FP64
# equivalent) and native launches (pack + GEMM) of the split-precision modes;
# FLOPs of the fp64 mode are counted the same way
STATS = {"flops": 0, "launches": 0, "gemms": 0}


def reset_stats():
    for k in STATS:
        STATS[k] = 0


def _dev_offsets(key, make, dev):
    t = _off_cache.get((key, dev))
    if t is None:
        t = torch.from_numpy(np.ascontiguousarray(make())).to(dev)
        if len(_off_cache) > 4096:
            _off_cache.clear()
        _off_cache[(key, dev)] = t
    return t


# ---- packed-operand cache ---------------------------------------------------------
# Operands whose storage was registered with mark_constant() keep their packed
# hi/lo arrays between calls (the MO integral blocks of the Lambda and CCSD
# iterations: vvvv alone is nvir^4 values).  The key holds every term's
# storage, offset, strides, shape, coefficient and torch version counter, so
# an in-place torch update of a registered tensor misses the cache; entries
# die with the registered tensor.
_const = {}                  # storage data_ptr -> weakref to the registered tensor
_pack_cache = {}             # key -> (hi, lo)
_PACK_CACHE_BYTES = 64 << 30
# switched off while a CUDA graph that is replayed with new operand values is
# captured: the graph must contain the packs, not read packs cached earlier
_PACK_CACHE_ON = [True]


class pack_cache_disabled:
    """Context manager: no packed-operand cache lookups or inserts inside."""

    def __enter__(self):
        self.prev = _PACK_CACHE_ON[0]
        _PACK_CACHE_ON[0] = False

    def __exit__(self, *exc):
        _PACK_CACHE_ON[0] = self.prev


def mark_constant(*tensors):
    """Declare tensors read-only for the rest of their life: contractions keep
    their split/packed forms instead of re-packing them on every call."""
    for t in tensors:
        if t is None or not isinstance(t, torch.Tensor) or t.device.type != "cuda":
            continue
        if torch._C._functorch.is_functorch_wrapped_tensor(t):
            continue                  # inside torch.func.vmap: no storage to key on
        ptr = t.untyped_storage().data_ptr()
        _const[ptr] = weakref.ref(t, lambda _r, ptr=ptr: _forget(ptr))


def _forget(ptr):
    _const.pop(ptr, None)
    for k in [k for k in _pack_cache if ptr in k[-1]]:
        del _pack_cache[k]


def clear_pack_cache():
    _pack_cache.clear()


def _is_const(t):
    r = _const.get(t.untyped_storage().data_ptr())
    return r is not None and r() is not None


def _cache_key(terms, sub, rows_idx, k_idx, shape_map, kind, rows_pad, k_pad):
    if not all(_is_const(t) for _, t in terms):
        return None
    desc = tuple((c, t.storage_offset(), tuple(t.stride()), tuple(t.shape), t._version) for c, t in terms)
    ptrs = tuple(t.untyped_storage().data_ptr() for _, t in terms)
    return (kind, rows_pad, k_pad, sub, tuple(rows_idx), tuple(k_idx),
            tuple(shape_map[i] for i in rows_idx + k_idx), desc, ptrs)


def _pack(terms, sub, rows_idx, k_idx, shape_map, kind, rows_pad, k_pad, dev, stream):
    key = _cache_key(terms, sub, rows_idx, k_idx, shape_map, kind, rows_pad, k_pad) if _PACK_CACHE_ON[0] else None
    if key is not None and key in _pack_cache:
        return _pack_cache[key]
    hi, lo = _pack_new(terms, sub, rows_idx, k_idx, shape_map, kind, rows_pad, k_pad, dev, stream)
    if key is not None:
        for k in [k for k in _pack_cache if k[:7] == key[:7] and k[-1] == key[-1]]:
            del _pack_cache[k]        # an older version of the same operand
        used = sum(h.numel() * 2 for h, _ in _pack_cache.values())
        if used + 2 * hi.numel() > _PACK_CACHE_BYTES:
            _pack_cache.clear()
        _pack_cache[key] = (hi, lo)
    return hi, lo


def _pack_new(terms, sub, rows_idx, k_idx, shape_map, kind, rows_pad, k_pad, dev, stream):
    rows = int(np.prod([shape_map[i] for i in rows_idx])) if rows_idx else 1
    K = int(np.prod([shape_map[i] for i in k_idx])) if k_idx else 1
    esz = 4 if kind == 0 else 2
    hi = torch.empty(rows_pad * k_pad * esz, dtype=torch.uint8, device=dev)
    lo = torch.empty_like(hi)
    offs = []
    for _, t in terms[:2]:
        key_r = ("r", tuple(rows_idx), sub, tuple(t.stride()), tuple(shape_map[i] for i in rows_idx))
        key_k = ("k", tuple(k_idx), sub, tuple(t.stride()), tuple(shape_map[i] for i in k_idx))
        offs.append((_dev_offsets(key_r, lambda t=t: _offsets(rows_idx, sub, shape_map, t), dev),
                     _dev_offsets(key_k, lambda t=t: _offsets(k_idx, sub, shape_map, t), dev)))
    (c1, t1), (o1r, o1k) = terms[0], offs[0]
    if len(terms) > 1:
        (c2, t2), (o2r, o2k) = terms[1], offs[1]
        p2 = (_native.ptr(t2), _native.ptr(o2r), _native.ptr(o2k), c2)
    else:
        p2 = (_native.ptr(None), _native.ptr(None), _native.ptr(None), 0.0)
    STATS["launches"] += 1
    # transposing gather: the source is contiguous along the packed rows
    st = dict(zip(sub, t1.stride()))
    sr = st.get(rows_idx[-1], 0) if rows_idx else 0
    sk = st.get(k_idx[-1], 0) if k_idx else 0
    rowfast = int(sr == 1 and sk != 1)
    _native.call("ccsd_b200_split_pack", kind, _native.ptr(t1), _native.ptr(o1r), _native.ptr(o1k), c1, *p2,
                 rows, K, rows_pad, k_pad, _native.ptr(hi), _native.ptr(lo), rowfast, stream)
    return hi, lo


# split-precision modes send a contraction to FP64 cuBLAS when its reduction
# is this short, or when its arithmetic intensity (FP64 flop per operand/result
# byte) is below LOW_INTENSITY_FLOP_PER_BYTE and K is at most
# LOW_INTENSITY_MAX_K: such shapes are bound by HBM, not by the tensor cores.
# Long, skinny reductions stay on the split-K tensor-core route (cuBLAS
# parallelises them poorly, and their large operands stay packed in the cache).
LOW_INTENSITY_K = 16
LOW_INTENSITY_FLOP_PER_BYTE = 12.0
LOW_INTENSITY_MAX_K = 1024
# below this many flops a contraction is launch-bound: one cuBLAS call beats
# two packs and a tensor-core launch, and FP64 is exact
SMALL_FLOPS = 5e7


# solvers whose largest contraction (the 2 o^2 v^4 ladder) is below this run
# in FP64: measured on ethanol/cc-pVDZ (4e9 flops: split precision 0.95x of
# FP64) and (H2O)3 (5e9: equal); (H2O)6 (3e11) gains 1.35x
MIXED_MIN_LADDER_FLOPS = 1e10


def effective_mode(mode, nocc, nvir):
    """The mode an iterative solver should run in.  Split precision gains
    nothing while the largest contraction is small: the packs and launches
    cost as much as the tensor cores save, and below SMALL_FLOPS every
    contraction takes the FP64 route anyway.  Such solves run in FP64
    directly (no split-precision phase, no FP64 polish)."""
    if mode != "fp64" and 2.0 * nocc * nocc * float(nvir) ** 4 < max(SMALL_FLOPS, MIXED_MIN_LADDER_FLOPS):
        return "fp64"
    return mode


def _combine(terms):
    (c, t), rest = terms[0], terms[1:]
    x = t * c if c != 1.0 or rest else t
    for c2, t2 in rest:
        x = x.add_(t2, alpha=c2)
    return x


# FP64 contractions whose largest operand exceeds this many bytes are done in
# slices of that operand along an output index (einsum may copy a permuted
# operand whole: 21.6 GB for the nvir 228 vvvv block)
_FP64_SLICE_BYTES = 4 << 30


def _fp64_sliced(spec, ta, tb, shape_map, out, alpha, beta):
    """The FP64 contraction with its largest operand cut into ~1 GB slices
    along an output index that only that operand carries; None when no slicing
    is needed or possible.  Each slice's einsum copies at most the slice."""
    na = max(t.numel() for _, t in ta)
    nb = max(t.numel() for _, t in tb)
    if max(na, nb) * 8 <= _FP64_SLICE_BYTES:
        return None
    sa, sb, so = _parse(spec)
    big_a = na >= nb
    sub_big, terms_big, sub_small = (sa, ta, sb) if big_a else (sb, tb, sa)
    ix = next((i for i in so if i in sub_big and i not in sub_small), None)
    if ix is None:
        return None
    n = shape_map[ix]
    chunk = max(1, int((1 << 30) // (8 * max(na, nb) / n)))
    if out is None:
        out = torch.empty([shape_map[i] for i in so], dtype=torch.float64, device=ta[0][1].device)
        beta = 0.0
    po, pb = so.index(ix), sub_big.index(ix)
    small = _combine(tb if big_a else ta)
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        big = _combine([(c, t.narrow(pb, c0, m)) for c, t in terms_big])
        res = torch.einsum(spec, big, small) if big_a else torch.einsum(spec, small, big)
        o = out.narrow(po, c0, m)
        if beta == 0.0:
            o.copy_(res * alpha if alpha != 1.0 else res)
        else:
            o.mul_(beta).add_(res, alpha=alpha)
    return out


def _fp64_contract(spec, ta, tb, shape_map, out, alpha, beta):
    """out = alpha * einsum(spec, a, b) + beta * out with torch.einsum (cuBLAS
    DGEMM); two-term operands are formed first, as the FP64 reference path does."""
    STATS["flops"] += 2 * int(np.prod(list(shape_map.values())))
    STATS["gemms"] += 1
    r = _fp64_sliced(spec, ta, tb, shape_map, out, alpha, beta)
    if r is not None:
        return r
    res = torch.einsum(spec, _combine(ta), _combine(tb))
    if beta == 0.0:
        out.copy_(res * alpha if alpha != 1.0 else res)
    else:
        out.mul_(beta).add_(res, alpha=alpha)
    return out


def contract(spec, a, b, out=None, alpha=1.0, beta=0.0, mode="tf32x3", stream=None):
    """out[...] = alpha * einsum(spec, a, b) + beta * out  (returns out)."""
    ta, tb = _terms(a), _terms(b)
    if len(ta) > 2 or len(tb) > 2:
        raise ValueError("an operand may have at most two terms")
    sa, sb, so = _parse(spec)
    shape_map = {}
    for sub, terms in ((sa, ta), (sb, tb)):
        for _, t in terms:
            if t.dim() != len(sub):
                raise ValueError("operand rank does not match %r" % spec)
            for ix, n in zip(sub, t.shape):
                if shape_map.setdefault(ix, n) != n:
                    raise ValueError("size mismatch for index %r in %r" % (ix, spec))
    dev = ta[0][1].device
    if mode == "fp64" and out is None:
        # no zero-filled output to copy into: also keeps the FP64 path free of
        # in-place writes, so it runs under torch.func.vmap (batched solves)
        STATS["flops"] += 2 * int(np.prod(list(shape_map.values())))
        STATS["gemms"] += 1
        r = _fp64_sliced(spec, ta, tb, shape_map, None, alpha, 0.0)
        if r is not None:
            return r
        res = torch.einsum(spec, _combine(ta), _combine(tb))
        return res * alpha if alpha != 1.0 else res
    if out is None:
        out = torch.zeros([shape_map[i] for i in so], dtype=torch.float64, device=dev)
        beta = 0.0
    if mode == "fp64":
        return _fp64_contract(spec, ta, tb, shape_map, out, alpha, beta)
    if mode not in KIND:
        raise ValueError("unknown mode %r" % mode)
    _native.require_cuda(out)
    batch = [i for i in so if i in sa and i in sb]
    if batch:
        ix = batch[0]
        for v in range(shape_map[ix]):
            sel = lambda sub, t: t.select(sub.index(ix), v)   # noqa: E731
            a_v = [(c, sel(sa, t)) for c, t in ta]
            b_v = [(c, sel(sb, t)) for c, t in tb]
            spec_v = "%s,%s->%s" % (sa.replace(ix, ""), sb.replace(ix, ""), so.replace(ix, ""))
            contract(spec_v, a_v, b_v, out=out.select(so.index(ix), v), alpha=alpha, beta=beta, mode=mode,
                     stream=stream)
        return out
    m_idx = [i for i in so if i in sa]
    n_idx = [i for i in so if i in sb]
    k_idx = [i for i in sa if i in sb and i not in so]
    for i in sa + sb:
        if i not in so and not (i in sa and i in sb):
            raise ValueError("index %r summed in one operand only: not a GEMM" % i)
    M = int(np.prod([shape_map[i] for i in m_idx])) if m_idx else 1
    N = int(np.prod([shape_map[i] for i in n_idx])) if n_idx else 1
    K = int(np.prod([shape_map[i] for i in k_idx])) if k_idx else 1
    if M == 0 or N == 0:
        return out
    # a registered constant operand stays packed in the cache, while the FP64
    # route would re-gather (permute-copy) it on every call
    big = ta if M >= N else tb
    big_cached = all(_is_const(t) for _, t in big)
    if K <= LOW_INTENSITY_K or 2.0 * M * N * K < SMALL_FLOPS or (
            not big_cached and K <= LOW_INTENSITY_MAX_K and
            2.0 * M * N * K < LOW_INTENSITY_FLOP_PER_BYTE * 8.0 * (M * K + N * K + M * N)):
        # memory-bound shape: FP64 through cuBLAS moves fewer bytes than the
        # split/pack/tensor-core route and is exact to FP64
        return _fp64_contract(spec, ta, tb, shape_map, out, alpha, beta)
    kind = KIND[mode]
    kal = _KALIGN[mode]
    m_pad, n_pad = M, N                    # tiles past M / N are zero-filled by TMA
    k_pad = max(kal, -(-K // kal) * kal)
    st = _native.stream(stream)
    ahi, alo = _pack(ta, sa, m_idx, k_idx, shape_map, kind, m_pad, k_pad, dev, st)
    bhi, blo = _pack(tb, sb, n_idx, k_idx, shape_map, kind, n_pad, k_pad, dev, st)
    key_m = ("om", tuple(m_idx), so, tuple(out.stride()), tuple(shape_map[i] for i in m_idx))
    key_n = ("on", tuple(n_idx), so, tuple(out.stride()), tuple(shape_map[i] for i in n_idx))
    om = _dev_offsets(key_m, lambda: _offsets(m_idx, so, shape_map, out), dev)
    on = _dev_offsets(key_n, lambda: _offsets(n_idx, so, shape_map, out), dev)
    kblocks = -(-k_pad // _KSTEP[mode])
    ksplit = _ksplit(m_pad, n_pad, kblocks, dev)
    if tune.gemm_tuning_active():
        def trial(s):
            scratch = torch.empty_strided(out.shape, out.stride(), dtype=torch.float64, device=dev)
            part = torch.empty(s * M * N, dtype=torch.float64, device=dev) if s > 1 else None
            _native.call("ccsd_b200_tc_split_gemm", kind, _native.ptr(ahi), _native.ptr(alo), _native.ptr(bhi),
                         _native.ptr(blo), M, N, m_pad, n_pad, k_pad, _native.ptr(scratch), _native.ptr(om),
                         _native.ptr(on), float(alpha), 0.0, s, _native.ptr(part), _native.ptr(_Status.get(dev)),
                         st)
        ksplit = tune.gemm_split(M, N, K, mode, ksplit, max(1, kblocks // _KB_PER_CHUNK), trial)
    partial = torch.empty(ksplit * M * N, dtype=torch.float64, device=dev) if ksplit > 1 else None
    STATS["flops"] += 2 * M * N * K
    STATS["gemms"] += 1
    STATS["launches"] += 1 if ksplit == 1 else 2
    _native.call("ccsd_b200_tc_split_gemm", kind, _native.ptr(ahi), _native.ptr(alo), _native.ptr(bhi),
                 _native.ptr(blo), M, N, m_pad, n_pad, k_pad, _native.ptr(out), _native.ptr(om), _native.ptr(on),
                 float(alpha), float(beta), ksplit, _native.ptr(partial), _native.ptr(_Status.get(dev)), st)
    return out


_sm_count = {}
_KB_PER_CHUNK = 16        # k blocks per FP32 accumulation chunk in the kernel (512 k)


def _ksplit(m_pad, n_pad, kblocks, dev):
    """Split-K factor: enough CTAs for two waves on the SMs when the output has
    few 128 x 128 tiles, with at least one 512-k chunk per split."""
    sms = _sm_count.get(dev)
    if sms is None:
        sms = _sm_count[dev] = torch.cuda.get_device_properties(dev).multi_processor_count
    tiles = -(-m_pad // _BM) * -(-n_pad // _BM)
    if tiles >= sms or kblocks < 2 * _KB_PER_CHUNK:
        return 1
    return int(max(1, min(-(-2 * sms // tiles), kblocks // _KB_PER_CHUNK)))
