"""Bounded-memory building blocks for large molecules.

The default chain keeps several dense (n,)*4 FP64 tensors resident at once
(the ERIs, the Coulomb-exchange matrix G of the SCF, four-index transform
temporaries, the AO 2-RDM and its Cartesian copy).  At n = 300 each is 65 GB,
so past n ~ 200 those paths no longer fit one B200.  The reference streams its
gradient by shell blocks sized from ``max_memory`` and blocks the Lambda over
the virtual index (ref: ccsd_gpu/gpu_ccsd_grad.py:416-432,
ccsd_gpu/gpu_ccsd_lambda.py:54-61).  Here the same goal is met with:

* four-index transforms blocked over the first output index
  (:func:`transform_rows`): the flop count of the unblocked transform, and no
  temporary larger than one block;
* an SCF that drops the cached G and builds J/K from the ERIs
  (:func:`jk_blocked`), an ao2mo that writes only the MO blocks the CC code
  reads, and a gradient that builds its two-electron density atom block by
  atom block (``gpu_ccsd_grad``), so that at most two (n,)*4 tensors are live.

:func:`lean` decides per call: on when the dense path would not fit the free
device memory, or when ``CCSD_B200_LOWMEM=1`` forces it (tests compare the
two paths on small molecules).
"""
import os

import torch

_FORCE = None


def force(on):
    """Force the bounded-memory paths on (True), off (False) or automatic (None)."""
    global _FORCE
    _FORCE = on


def lean(n_tensors, n, device=None, dtype_bytes=8):
    """True when ``n_tensors`` dense (n,)*4 tensors would not fit in 85% of
    the free device memory (or when forced)."""
    if _FORCE is not None:
        return bool(_FORCE)
    if os.environ.get("CCSD_B200_LOWMEM") == "1":
        return True
    need = n_tensors * float(n) ** 4 * dtype_bytes
    if need < 1e9:                      # small molecules: no query at all
        return False
    # the allocator's own counters (no driver call, no synchronisation): the
    # device's memory minus what torch holds, less a margin for the context
    # and library workspaces
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else device
    free = _total(dev) - torch.cuda.memory_allocated(dev) - (4 << 30)
    return need > 0.85 * free


_TOTAL = {}


def _total(dev):
    key = dev.index if dev.index is not None else torch.cuda.current_device()
    if key not in _TOTAL:
        _TOTAL[key] = torch.cuda.get_device_properties(key).total_memory
    return _TOTAL[key]


def tidy(n, device=None):
    """Hand the allocator's cached free blocks back to the device when the
    dense paths do not fit (n: AO count), so the next stage's large tensors
    get fresh segments instead of failing on a fragmented cache."""
    if lean(4, n, device):
        torch.cuda.empty_cache()


def block_size(n, rows_budget_bytes=2 << 30, dtype_bytes=8):
    """Rows per block of a first-index-blocked (n,)*4 transform: about
    rows_budget_bytes of (rows, n, n, n) per block, at least one row."""
    return max(1, int(rows_budget_bytes // (dtype_bytes * float(n) ** 3)))


def transform_rows(T, Cp, Cq, Cr, Cs):
    """out[p, q, r, s] = sum_{abcd} Cp[a, p] Cq[b, q] Cr[c, r] Cs[d, s] T[a, b, c, d]
    for the columns p of Cp (one block of the output's first index).

    T is (na, nb, nc, nd), contiguous.  The first step is one GEMM on T as it
    lies; the other three act on the block-sized result, so no temporary is
    larger than a block."""
    na, nb, nc, nd = T.shape
    x = (Cp.T @ T.reshape(na, nb * nc * nd)).reshape(Cp.shape[1], nb, nc, nd)
    return torch.einsum("pbcd,bq,cr,ds->pqrs", x, Cq, Cr, Cs)


def transform_cols1(T, Cp, Cq_blk, Cr, Cs):
    """The same transform for a block of the SECOND output index (the columns
    q of Cq_blk), returned as (q, p, r, s): the transposed slab that the
    (p <-> q) symmetrisation of a row block needs.  The first step contracts b
    for every a (a batched GEMM on T as it lies)."""
    na, nb, nc, nd = T.shape
    x = torch.matmul(Cq_blk.T, T.reshape(na, nb, nc * nd)).reshape(na, Cq_blk.shape[1], nc, nd)   # (a, q, c, d)
    return torch.einsum("aqcd,ap,cr,ds->qprs", x, Cp, Cr, Cs)


def transform_all(T, C, block=None):
    """Full four-index transform with one matrix, blocked over the first
    output index: returns sum C[a,p] C[b,q] C[c,r] C[d,s] T[a,b,c,d]; T is
    freed by the caller once this returns (only T, the output and one block
    are ever live)."""
    n_out = C.shape[1]
    out = torch.empty((n_out,) * 4, dtype=T.dtype, device=T.device)
    bs = block or block_size(max(T.shape[0], n_out))
    for p0 in range(0, n_out, bs):
        p1 = min(n_out, p0 + bs)
        out[p0:p1] = transform_rows(T, C[:, p0:p1], C, C, C)
    return out


def jk_blocked(eri, dm, block=None):
    """(J, K) of a density from the dense chemist-notation ERIs,
    J[p,q] = sum (pq|rs) D[r,s], K[p,q] = sum (pr|qs) D[r,s], with the exchange
    contraction done block by block over p (no permuted copy of the ERIs)."""
    n = dm.shape[0]
    J = (eri.reshape(n * n, n * n) @ dm.reshape(n * n)).reshape(n, n)
    K = torch.empty_like(dm)
    bs = block or max(1, block_size(n) // 2)
    for p0 in range(0, n, bs):
        p1 = min(n, p0 + bs)
        # (p, r, q, s) rows of the block; K[p, q] = sum_{r s} eri[p, r, q, s] D[r, s]
        blk = eri[p0:p1]                                          # (p, r, q, s)
        K[p0:p1] = torch.einsum("prqs,rs->pq", blk, dm)
    return J, K
