"""CCSD gradients of many molecules of uneven size (the batched workload).

``gradients(mols, precision, polish=False, batched=True)`` returns the
gradient dE/dR (natm, 3) of every molecule, in input order.  The reference
computes one molecule per run (examples/h2o_ccsd_grad.py:100-166); here the
molecules are grouped by shape (nao, nocc, nvir) and each group is solved in
lockstep:

  * RHF and the AO->MO transform per molecule;
  * the T-amplitude and Lambda iterations of a whole group as one batched
    body: the per-molecule update (``update_amps_gpu``, the Lambda
    intermediates and ``update_lambda_gpu``) is mapped over the group with
    ``torch.func.vmap`` -- every contraction becomes one batched GEMM over
    the molecules -- and captured once per (shape, group size) as a CUDA
    graph that later groups of the same shape replay.  Norms, energies and
    the DIIS extrapolation are batched over the group on the device; the host
    reads one vector of update norms per iteration for the convergence test.
    A molecule that has converged keeps its amplitudes.
  * the gradient assembly per molecule (``grad_elec_gpu``), from the device
    amplitudes of the batched solves.

Batching applies to shapes whose solves run in FP64 in every mode (the 2 o^2
v^4 ladder below ``contract.MIXED_MIN_LADDER_FLOPS``): there a solve is bound
by launch latency and host work, which the batched graph pays once per group
instead of once per molecule.  Larger shapes fill the GPU one molecule at a
time and go through the per-molecule chain (split-precision contractions are
native tensor-core calls, which vmap does not batch).
"""
from types import SimpleNamespace

import numpy as np
import torch

from .contract import MIXED_MIN_LADDER_FLOPS, SMALL_FLOPS, check_status, effective_mode
from .gpu_ccsd_lambda import DeviceEris, host_copy, make_intermediates_gpu, remember_device, update_lambda_gpu

_ERI_KEYS = ("fock", "mo_energy", "oooo", "ovoo", "ovvo", "oovv", "ovov", "ovvv", "vvvv")


def batchable(nocc, nvir):
    """Shapes solved in lockstep: the ones whose solves run in FP64 in every mode."""
    return 2.0 * nocc * nocc * float(nvir) ** 4 < max(SMALL_FLOPS, MIXED_MIN_LADDER_FLOPS)


def _eris_of(consts):
    """A DeviceEris over already-resident (possibly batched) tensors."""
    e = object.__new__(DeviceEris)
    e.__dict__.update({k: consts[k] for k in _ERI_KEYS})
    e.nocc = consts["ovoo"].shape[0]
    return e


def _energy(t1, t2, eris):
    nocc = t1.shape[0]
    tau = t2 + torch.einsum("ia,jb->ijab", t1, t1)
    ov = eris.ovov
    return (2 * (eris.fock[:nocc, nocc:] * t1).sum() + 2 * torch.einsum("ijab,iajb->", tau, ov)
            - torch.einsum("ijab,ibja->", tau, ov))


def _norm_sq(d1, d2):
    nocc, nvir = d1.shape
    m = d2.permute(0, 2, 1, 3).reshape(nocc * nvir, nocc * nvir)
    return (d1 * d1).sum() + 0.5 * ((m * m).sum() + (torch.diagonal(m) ** 2).sum())


def _t_body(consts, t1, t2):
    from .ccsd import update_amps_gpu
    return update_amps_gpu(t1, t2, _eris_of(consts), "fp64", 0.0)


def _l_body(consts, l1, l2):
    imds = SimpleNamespace(mode="fp64", **{k: consts["i_" + k] for k in _IMDS})
    return update_lambda_gpu(SimpleNamespace(level_shift=0.0), consts["t1"], consts["t2"], l1, l2,
                             _eris_of(consts), imds, mode="fp64")


def _imds_body(consts):
    im = make_intermediates_gpu(SimpleNamespace(level_shift=0.0), consts["t1"], consts["t2"], _eris_of(consts),
                                "fp64")
    return tuple(getattr(im, k) for k in _IMDS)


_IMDS = ("w1", "w2", "w3", "w4", "woooo", "wvooo", "wVOov", "wvOOv", "wvvov")


def _energy_c(consts, t1, t2):
    return _energy(t1, t2, _eris_of(consts))


class _BatchDIIS:
    """Pulay extrapolation of B independent solves at once (FP64, device),
    error vector = x_new - x_old; ring buffers and incrementally updated Gram
    matrices, as the per-molecule DIIS of the solvers."""

    def __init__(self, B, n, space, dev):
        self.space, self.count = space, 0
        self.xbuf = torch.empty((B, space, n), dtype=torch.float64, device=dev)
        self.ebuf = torch.empty_like(self.xbuf)
        self.gram = torch.zeros((B, space, space), dtype=torch.float64, device=dev)

    def update(self, x, err):
        slot = self.count % self.space
        self.count += 1
        m = min(self.count, self.space)
        self.xbuf[:, slot] = x
        self.ebuf[:, slot] = err
        row = torch.bmm(self.ebuf[:, :m], err[:, :, None])[:, :, 0]
        self.gram[:, slot, :m] = row
        self.gram[:, :m, slot] = row
        if m < 2:
            return x
        B = x.shape[0]
        G = self.gram[:, :m, :m]
        scale = G.diagonal(dim1=1, dim2=2).abs().amax(1).clamp_min(1e-300)
        A = torch.empty((B, m + 1, m + 1), dtype=torch.float64, device=x.device)
        A[:, :m, :m] = G / scale[:, None, None]
        A[:, m, :m] = -1.0
        A[:, :m, m] = -1.0
        A[:, m, m] = 0.0
        rhs = torch.zeros((B, m + 1, 1), dtype=torch.float64, device=x.device)
        rhs[:, m] = -1.0
        c = torch.linalg.lstsq(A, rhs).solution[:, :m, 0]
        return torch.bmm(c[:, None, :], self.xbuf[:, :m])[:, 0]


class _GroupGraph:
    """``vmap(fn)(consts, *inputs)`` over a group, captured as one CUDA graph.

    The first call runs eagerly and captures; the graph is kept per key, and a
    later group of the same shape and size copies its constants in and
    replays it."""

    def __init__(self, fn, consts, inputs):
        self.fn = torch.func.vmap(fn)
        self.consts = {k: v.detach().clone() for k, v in consts.items()}
        self.static_in = [x.detach().clone() for x in inputs]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.fn(self.consts, *self.static_in)
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.static_out = tuple(self.fn(self.consts, *self.static_in))

    def load(self, consts):
        for k, v in consts.items():
            self.consts[k].copy_(v)

    def __call__(self, *inputs):
        for d, x in zip(self.static_in, inputs):
            d.copy_(x)
        self.graph.replay()
        return tuple(o.clone() for o in self.static_out)


_GRAPHS = {}
_GRAPHS_MAX = 16


def _group_step(key, fn, consts, inputs):
    key = (torch.cuda.current_device(),) + tuple(key)
    g = _GRAPHS.get(key)
    if g is None:
        g = _GroupGraph(fn, consts, inputs)
        if len(_GRAPHS) >= _GRAPHS_MAX:
            _GRAPHS.pop(next(iter(_GRAPHS)))
        _GRAPHS[key] = g
    else:
        g.load(consts)
    return g


def clear_graphs():
    _GRAPHS.clear()


def _flat(t1, t2):
    return torch.cat([t1.reshape(t1.shape[0], -1), t2.reshape(t2.shape[0], -1)], 1)


def _solve_group(ccs, lambda_tol):
    """T amplitudes and Lambda of every CC object of one shape group, in lockstep."""
    dev = torch.device("cuda", torch.cuda.current_device())
    eris = [cc.ao2mo() for cc in ccs]
    B = len(ccs)
    nocc = ccs[0].nocc
    consts = {k: torch.stack([getattr(e, k) for e in eris]) for k in _ERI_KEYS}
    nvir = consts["fock"].shape[1] - nocc
    eo, ev = consts["mo_energy"][:, :nocc], consts["mo_energy"][:, nocc:]
    eia = eo[:, :, None] - ev[:, None, :]
    d2 = eia[:, :, None, :, None] + eia[:, None, :, None, :]
    t1 = consts["fock"][:, :nocc, nocc:] / eia
    t2 = consts["ovov"].permute(0, 1, 3, 2, 4) / d2
    n1 = nocc * nvir
    norm = torch.func.vmap(_norm_sq)
    energy = torch.func.vmap(_energy_c)
    # ---- T amplitudes (the per-molecule solver's tolerances)
    conv_tol, tol_n = ccs[0].conv_tol, ccs[0].conv_tol_normt
    step = _group_step(("T", B, nocc, nvir), _t_body, consts, (t1, t2))
    diis = _BatchDIIS(B, t1[0].numel() + t2[0].numel(), ccs[0].diis_space, dev)
    e_old = energy(consts, t1, t2)
    done = torch.zeros(B, dtype=torch.bool, device=dev)
    hist = []
    for it in range(max(cc.max_cycle for cc in ccs)):
        t1n, t2n = step(t1, t2)
        nt = torch.sqrt(norm(t1n - t1, t2n - t2))
        x = diis.update(_flat(t1n, t2n), _flat(t1n - t1, t2n - t2))
        keep = done[:, None]
        x = torch.where(keep, _flat(t1, t2), x)
        t1, t2 = x[:, :n1].reshape(t1.shape), x[:, n1:].reshape(t2.shape)
        e = energy(consts, t1, t2)
        ok = (nt < tol_n) & ((e - e_old).abs() < conv_tol)
        done = done | ok
        e_old = e
        host = torch.stack([nt, done.double()]).cpu().numpy()
        hist.append(host[0])
        if host[1].all():
            break
    e = e_old.cpu().numpy()
    for b, cc in enumerate(ccs):
        cc.converged = bool(host[1][b])
        cc.normt = float(host[0][b])
        cc._t_history = [("fp64", float(h[b])) for h in hist]
        cc.e_corr = float(e[b])
        cc.t1, cc.t2 = host_copy(t1[b]), host_copy(t2[b])
        remember_device(cc, "t1", cc.t1, t1[b].clone())
        remember_device(cc, "t2", cc.t2, t2[b].clone())
    # ---- Lambda: intermediates for the whole group, then lockstep updates
    lc = dict(consts, t1=t1, t2=t2)
    imds = torch.func.vmap(_imds_body)(lc)
    lc.update({"i_" + k: v for k, v in zip(_IMDS, imds)})
    del imds
    l1, l2 = t1.clone(), t2.clone()
    step = _group_step(("L", B, nocc, nvir), _l_body, lc, (l1, l2))
    diis = _BatchDIIS(B, l1[0].numel() + l2[0].numel(), ccs[0].diis_space, dev)
    done = torch.zeros(B, dtype=torch.bool, device=dev)
    hist = []
    for it in range(max(cc.max_cycle for cc in ccs)):
        l1n, l2n = step(l1, l2)
        nt = torch.sqrt(norm(l1n - l1, l2n - l2))
        x = diis.update(_flat(l1n, l2n), _flat(l1n - l1, l2n - l2))
        x = torch.where(done[:, None], _flat(l1, l2), x)
        l1, l2 = x[:, :n1].reshape(l1.shape), x[:, n1:].reshape(l2.shape)
        done = done | (nt < lambda_tol)
        host = torch.stack([nt, done.double()]).cpu().numpy()
        hist.append(host[0])
        if host[1].all():
            break
    for b, cc in enumerate(ccs):
        cc.converged_lambda = bool(host[1][b])
        cc.lambda_normt = float(host[0][b])
        cc._lambda_history = [("fp64", float(h[b])) for h in hist]
        cc.l1, cc.l2 = host_copy(l1[b]), host_copy(l2[b])
        remember_device(cc, "l1", cc.l1, l1[b].clone())
        remember_device(cc, "l2", cc.l2, l2[b].clone())
        cc._lambda_solver_mode = "gpu-batched-fp64"
    check_status()


def gradients(mols, precision="tf32x3", polish=False, batched=True, lambda_tol=1e-9):
    """dE/dR (natm, 3) numpy per molecule, electronic + nuclear, in input order.

    ``precision``: the CC objects' mode; ``polish``: the FP64 refinement of
    split-precision solves; ``batched=False`` solves one molecule after the
    other (same chain as ``CCSD(RHF(mol).run()).nuc_grad_method().kernel()``).
    Shape groups are processed one at a time, so at most one group's
    integrals are resident."""
    from .ccsd import CCSD
    from .scf import RHF
    out = [None] * len(mols)
    groups = {}
    for i, mol in enumerate(mols):
        groups.setdefault((mol.nao_nr(), mol.nelectron // 2), []).append(i)

    def make_cc(mol):
        cc = CCSD(RHF(mol).run(), precision=precision)
        cc.t_polish = cc.lambda_polish = bool(polish)
        return cc

    for (nao, nocc), idx in groups.items():
        nvir = nao - nocc
        if batched and len(idx) > 1 and batchable(nocc, nvir) and effective_mode(precision, nocc, nvir) == "fp64":
            ccs = [make_cc(mols[i]) for i in idx]
            _solve_group(ccs, lambda_tol)
            for i, cc in zip(idx, ccs):
                cc.conv_tol_normt = lambda_tol
                out[i] = cc.nuc_grad_method().kernel()
            del ccs
        else:
            for i in idx:
                cc = make_cc(mols[i])
                cc.kernel()
                cc.conv_tol_normt = lambda_tol
                out[i] = cc.nuc_grad_method().kernel()
                del cc
    return out
