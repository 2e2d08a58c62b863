"""CCSD Lambda (l1, l2) solver on the GPU.

Drop-in for ``ccsd_gpu.gpu_ccsd_lambda`` (ref: ccsd_gpu/gpu_ccsd_lambda.py):
``make_intermediates_gpu`` (:68-209), ``update_lambda_gpu`` (:212-337),
``kernel_gpu`` (:340-408) and ``solve_lambda_gpu`` (:411-449) keep their
signatures.  Differences from the reference:

  * every contraction runs through :func:`ccsd_gpu_b200.contract.contract`:
    split-precision tcgen05 GEMMs (``"tf32x3"``, the default, or ``"bf16x3"``)
    or plain FP64 (``"fp64"``, cuBLAS) -- chosen with the ``precision``
    attribute of the CC object or the ``mode`` keyword;
  * the vvvv ladder sum_cd l2[ijcd] (ac|bd) runs on the GPU (the reference
    calls PySCF's CPU ``_add_vvvv``); ``use_cpu_vvvv`` is accepted and ignored;
  * the amplitude norm and the DIIS extrapolation stay FP64 and on the device
    (the reference copies four amplitude sets to the host every iteration);
  * there is no CPU path: ``fallback_to_cpu`` is accepted, and without a
    usable GPU the solver raises.
The equations are PySCF's closed-shell RCCSD Lambda equations, the same index
equations the reference evaluates (checked against its output in tests/).
"""
from types import SimpleNamespace

import numpy as np
import torch

from . import _native
from .contract import check_status, contract, effective_mode, mark_constant
from .graphs import StepGraph, graph_cache_ok, solve_step

DEFAULT_MODE = "tf32x3"


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def _t(x, dev=None):
    if isinstance(x, torch.Tensor):
        return x.to(dev or _dev(), dtype=torch.float64)
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=dev or _dev())


class DeviceEris:
    """MO integral blocks (chemist notation, PySCF layout) resident on the GPU."""

    def __init__(self, eris, dev=None):
        dev = dev or _dev()
        self.fock = _t(eris.fock, dev)
        self.mo_energy = _t(eris.mo_energy, dev)
        for k in ("oooo", "ovoo", "ovvo", "oovv", "ovov"):
            setattr(self, k, _t(getattr(eris, k), dev))
        ovvv = getattr(eris, "ovvv", None)
        if ovvv is None or getattr(ovvv, "ndim", 4) != 4:
            ovvv = eris.get_ovvv(slice(None))
        self.ovvv = _t(ovvv, dev)
        self.vvvv = _t(eris.vvvv, dev) if getattr(eris, "vvvv", None) is not None else None
        self.nocc = self.ovoo.shape[0]
        mark_constant(self.oooo, self.ovoo, self.ovvo, self.oovv, self.ovov, self.ovvv, self.vvvv)

    @classmethod
    def wrap(cls, eris):
        return eris if isinstance(eris, cls) else cls(eris)


def host_copy(x):
    """Read-only numpy copy of the device tensor ``x``, read into pinned host
    memory (torch's caching host allocator reuses the block once the array is
    dropped; a pageable read of a 100 MB amplitude runs at ~4 GB/s)."""
    h = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
    h.copy_(x)
    a = h.numpy()
    a.setflags(write=False)
    return a


def remember_device(mycc, name, host, dev):
    """Record that the host array ``mycc.<name>`` (``host``) has the device
    copy ``dev``, so later steps of the chain skip the round trip.  ``host``
    is read-only (``host_copy``), so the pair cannot drift apart."""
    d = mycc.__dict__.setdefault("_dev_amps", {})
    d[name] = (host, dev)


def device_amp(mycc, name, value):
    """The device copy of ``value`` if it is the array this package produced
    for ``mycc.<name>`` (identity check), else ``value`` itself."""
    d = getattr(mycc, "_dev_amps", {}).get(name)
    return d[1] if d is not None and d[0] is value else value


class _Ctx:
    """Contraction helper bound to one precision mode."""

    def __init__(self, mode):
        self.mode = mode

    def __call__(self, spec, a, b, out=None, alpha=1.0, beta=0.0):
        return contract(spec, a, b, out=out, alpha=alpha, beta=beta, mode=self.mode)


def _mode_of(mycc, mode):
    return mode or getattr(mycc, "precision", None) or DEFAULT_MODE


def make_intermediates_gpu(mycc, t1, t2, eris, mode=None):
    """Lambda intermediates (ref: ccsd_gpu/gpu_ccsd_lambda.py:68-209)."""
    _native.require_cuda()
    E = _Ctx(_mode_of(mycc, mode))
    eris = DeviceEris.wrap(eris)
    t1, t2 = _t(t1), _t(t2)
    nocc, nvir = t1.shape
    fock = eris.fock
    foo, fov, fvv = fock[:nocc, :nocc], fock[:nocc, nocc:], fock[nocc:, nocc:]
    ovvv, ovoo, ovvo, oovv, oooo = eris.ovvv, eris.ovoo, eris.ovvo, eris.oovv, eris.oooo
    vvov = ovvv.permute(2, 3, 0, 1)
    voov = ovvo.permute(1, 0, 3, 2)
    t2T = t2.permute(1, 0, 2, 3)
    tau = t2 + torch.einsum("ia,jb->ijab", t1, t1)
    theta_b = [(2.0, t2), (-1.0, t2T)]                     # 2 t2[ijab] - t2[jiab]
    theta_c = [(2.0, t2), (-1.0, t2.permute(0, 1, 3, 2))]  # 2 t2[ijab] - t2[ijba]
    # one-particle intermediates
    w1 = fvv - t1.T @ fov
    w2 = foo + fov @ t1.T
    w3 = fov.T.clone(memory_format=torch.contiguous_format)
    E("kc,jkbc->bj", fov, theta_b, out=w3, beta=1.0)
    w3 += torch.einsum("kc,kb,jc->bj", fov, t1, t1)
    E("jcba,jc->ba", ovvv, t1, out=w1, alpha=2.0, beta=1.0)
    E("jabc,jc->ba", ovvv, t1, out=w1, alpha=-1.0, beta=1.0)
    E("jkcd,kdcb->bj", theta_b, ovvv, out=w3, beta=1.0)
    E("kbij,kb->ij", ovoo, t1, out=w2, alpha=2.0, beta=1.0)
    E("ibkj,kb->ij", ovoo, t1, out=w2, alpha=-1.0, beta=1.0)
    E("lckj,klcb->bj", ovoo, [(2.0, t2T), (-1.0, t2)], out=w3, alpha=-1.0, beta=1.0)
    g2voov = [(2.0, voov), (-1.0, voov.permute(0, 2, 1, 3))]
    x4 = E("ckld,ld->kc", g2voov, t1)
    E("ckja,kjcb->ba", g2voov, t2, out=w1, alpha=-1.0, beta=1.0)
    w1 -= t1.T @ x4
    E("jkbc,bikc->ij", t2, g2voov, out=w2, beta=1.0)
    w2 += x4 @ t1.T
    w3 += t1.T @ x4 @ t1.T
    w4 = fov + x4
    # two-particle intermediates
    VOov = voov.clone(memory_format=torch.contiguous_format)
    E("bjld,klcd->bjkc", g2voov, t2, out=VOov, beta=1.0)
    E("bjld,kldc->bjkc", voov, t2, out=VOov, alpha=-1.0, beta=1.0)
    vOOv = (-oovv.permute(2, 1, 0, 3)).contiguous()
    E("bljd,kldc->bjkc", voov, t2, out=vOOv, beta=1.0)
    t1t1 = torch.einsum("kd,lc->kldc", t1, t1)
    wVOov = VOov.clone()
    E("jbcd,kd->bjkc", ovvv, t1, out=wVOov, beta=1.0)
    E("jbkl,lc->bjkc", ovoo, t1, out=wVOov, alpha=-1.0, beta=1.0)
    E("bjld,kldc->bjkc", voov, t1t1, out=wVOov, alpha=-1.0, beta=1.0)
    wvOOv = vOOv.clone()
    E("cbjd,kd->cjkb", vvov, t1, out=wvOOv, alpha=-1.0, beta=1.0)
    E("lbjk,lc->bjkc", ovoo, t1, out=wvOOv, beta=1.0)
    E("bljd,kldc->bjkc", voov, t1t1, out=wvOOv, beta=1.0)
    ov1 = 2 * vOOv + VOov
    ov2 = 2 * VOov + vOOv
    x = E("lc,jcik->ijkl", t1, ovoo)
    woooo = x + x.permute(1, 0, 3, 2) + oooo.permute(0, 2, 1, 3)
    E("cijd,klcd->ijkl", voov, tau, out=woooo, beta=1.0)
    g2vovv = [(2.0, vvov.permute(0, 2, 1, 3)), (-1.0, vvov.permute(0, 2, 3, 1))]
    g2ovoo = [(2.0, ovoo), (-1.0, ovoo.permute(2, 1, 0, 3))]
    vcjik = E("jlcb,lbki->cjki", theta_b, g2ovoo)
    wvooo = (2 * ovoo.permute(1, 3, 2, 0) - ovoo.permute(1, 0, 2, 3)
             + vcjik.permute(0, 3, 2, 1) - 0.5 * vcjik).contiguous()
    E("cibd,jkbd->ckij", g2vovv, tau, out=wvooo, beta=1.0)
    E("klbc,iblj->ckij", t2, ovoo, out=wvooo, alpha=-1.5, beta=1.0)
    E("jb,bikc->ckij", t1, ov1, out=wvooo, alpha=-1.0, beta=1.0)
    E("kb,bijc->ckij", t1, ov2, out=wvooo, beta=1.0)
    g2vvov = [(2.0, vvov), (-1.0, ovvv.permute(1, 2, 0, 3))]
    vackb = E("acjd,kjbd->ackb", g2vvov, theta_c)
    wvvov = (2 * vvov.permute(0, 3, 2, 1) - vvov + vackb.permute(0, 3, 2, 1) - 0.5 * vackb).contiguous()
    del vackb
    E("jabd,jkcd->abkc", ovvv, t2, out=wvvov, alpha=-1.5, beta=1.0)
    E("ajkc,jb->abkc", ov1, t1, out=wvvov, beta=1.0)
    E("ajkb,jc->abkc", ov2, t1, out=wvvov, alpha=-1.0, beta=1.0)
    E("laki,klbc->abic", g2ovoo, tau, out=wvvov, beta=1.0)
    E("ckjb,kc->bj", ov2, t1, out=w3, beta=1.0)
    w3 += w1 @ t1.T - t1.T @ w2
    mark_constant(woooo, wvooo, wVOov, wvOOv, wvvov)
    return SimpleNamespace(w1=w1, w2=w2, w3=w3, w4=w4, woooo=woooo, wvooo=wvooo, wVOov=wVOov, wvOOv=wvOOv,
                           wvvov=wvvov, mode=E.mode)


def update_lambda_gpu(mycc, t1, t2, l1, l2, eris=None, imds=None, use_cpu_vvvv=True, mode=None):
    """One Jacobi update of (l1, l2) (ref: ccsd_gpu/gpu_ccsd_lambda.py:212-337)."""
    _native.require_cuda()
    eris = DeviceEris.wrap(eris)
    if imds is None:
        imds = make_intermediates_gpu(mycc, t1, t2, eris, mode)
    E = _Ctx(mode or imds.mode)
    t1, t2, l1, l2 = _t(t1), _t(t2), _t(l1), _t(l2)
    nocc, nvir = t1.shape
    fov = eris.fock[:nocc, nocc:]
    eo = eris.mo_energy[:nocc]
    ev = eris.mo_energy[nocc:] + float(getattr(mycc, "level_shift", 0.0))
    ovvv, ovoo, ovvo, oovv = eris.ovvv, eris.ovoo, eris.ovvo, eris.oovv
    voov = ovvo.permute(1, 0, 3, 2)
    theta = [(2.0, t2), (-1.0, t2.permute(0, 1, 3, 2))]
    mba = E("klca,klcb->ba", l2, theta)
    mij = E("ikcd,jkcd->ij", l2, theta)
    mba1 = t1.T @ l1 + mba
    mij1 = l1 @ t1.T + mij
    mia1 = t1 - t1 @ l1.T @ t1 - t1 @ mba.T - mij.T @ t1
    E("kc,jkbc->jb", l1, theta, out=mia1, beta=1.0)
    # vvvv ladder on the tensor cores: l2n = 0.5 sum_cd l2[ijcd] (ac|bd)
    l2n = E("ijcd,acbd->ijab", l2, eris.vvvv, alpha=0.5)
    l1n = E("ijab,jb->ia", [(4.0, l2n), (-2.0, l2n.permute(1, 0, 2, 3))], t1)
    w1 = imds.w1 - torch.diag(ev)
    w2 = imds.w2 - torch.diag(eo)
    l1n += fov + l1 @ w1 - w2 @ l1 - mij @ imds.w4 - imds.w4 @ mba
    E("ijab,bj->ia", [(2.0, l2), (-1.0, l2.permute(0, 1, 3, 2))], imds.w3, out=l1n, beta=1.0)
    l2n += torch.einsum("ia,jb->ijab", l1, imds.w4)
    E("jibc,ca->jiba", l2, w1, out=l2n, beta=1.0)
    E("jk,kiba->jiba", w2, l2, out=l2n, alpha=-1.0, beta=1.0)
    E("iajk,kj->ia", [(2.0, ovoo), (-1.0, ovoo.permute(2, 1, 0, 3))], mij1, out=l1n, alpha=-1.0, beta=1.0)
    E("jbki,ka->jiba", ovoo, l1, out=l2n, alpha=-1.0, beta=1.0)
    tau = t2 + torch.einsum("ia,jb->ijab", t1, t1)
    l2tau = E("ijcd,klcd->ijkl", l2, tau)
    l2t1 = E("jidc,kc->ijkd", l2, t1)
    E("jb,jiab->ia", l1, oovv, out=l1n, alpha=-1.0, beta=1.0)
    E("iabc,bc->ia", [(2.0, ovvv), (-1.0, ovvv.permute(0, 3, 1, 2))], mba1, out=l1n, beta=1.0)
    E("jbac,ic->jiba", ovvv, l1, out=l2n, beta=1.0)
    m4 = E("ijkd,kadb->ijab", l2t1, ovvv)
    l2n -= m4
    m4c = [(2.0, m4), (-1.0, m4.permute(1, 0, 2, 3))]
    E("ijab,jb->ia", m4c, t1, out=l1n, alpha=-1.0, beta=1.0)
    E("ijab,ia->jb", m4c, t1, out=l1n, alpha=-1.0, beta=1.0)
    E("jb,aijb->ia", l1, voov, out=l1n, alpha=2.0, beta=1.0)
    l2n += 0.5 * voov.permute(1, 2, 0, 3)
    E("bjic,ca->jiba", voov, mba1, out=l2n, alpha=-1.0, beta=1.0)
    E("bjka,ik->jiba", voov, mij1, out=l2n, alpha=-1.0, beta=1.0)
    E("aijb,jb->ia", [(2.0, voov), (-1.0, voov.permute(3, 1, 2, 0))], mia1, out=l1n, beta=1.0)
    m4 = E("ijkl,aklb->ijab", l2tau, voov)
    l2n += 0.5 * m4
    E("ijab,jb->ia", [(2.0, m4), (-1.0, m4.permute(0, 1, 3, 2))], t1, out=l1n, beta=1.0)
    E("ckij,jkca->ia", imds.wvooo, l2, out=l1n, alpha=-1.0, beta=1.0)
    E("abkc,kibc->ia", imds.wvvov, l2, out=l1n, beta=1.0)
    E("iakc,bjkc->jiba", [(1.0, l2.permute(0, 2, 1, 3)), (-0.5, l2.permute(0, 3, 1, 2))],
      [(2.0, imds.wVOov), (1.0, imds.wvOOv)], out=l2n, beta=1.0)
    tmp = E("jkca,bikc->jiba", l2, imds.wvOOv)
    l2n += tmp + 0.5 * tmp.permute(1, 0, 2, 3)
    m3 = E("ijkl,klab->ijab", imds.woooo, l2)
    l2n += 0.5 * m3
    E("ijab,jb->ia", [(2.0, m3), (-1.0, m3.permute(0, 1, 3, 2))], t1, out=l1n, beta=1.0)
    eia = eo[:, None] - ev[None, :]
    l1n /= eia
    l2n = (l2n + l2n.permute(1, 0, 3, 2)) / (eia[:, None, :, None] + eia[None, :, None, :])
    return l1n, l2n


def amplitude_norm_sq(d1, d2):
    """|d1|^2 + |lower triangle (incl. diagonal) of d2 as the (ia, jb) matrix|^2 --
    the norm of PySCF's RCCSD amplitude vector."""
    nocc, nvir = d1.shape
    m = d2.permute(0, 2, 1, 3).reshape(nocc * nvir, nocc * nvir)
    return (d1 * d1).sum() + 0.5 * ((m * m).sum() + (torch.diagonal(m) ** 2).sum())


class DIIS:
    """Pulay extrapolation on the device in FP64; error vector = x_new - x_old.

    The vectors live in two preallocated ring buffers and the Gram matrix of
    the error vectors is kept up to date, so one update reads the stored
    errors once (one GEMV for the new row of the Gram matrix) and the stored
    vectors once (one GEMV for the extrapolation): no stacking copies and no
    Gram GEMM over the whole subspace per iteration."""

    def __init__(self, space=6):
        self.space = space
        self.count = 0
        self.xbuf = self.ebuf = self.gram = None

    def update(self, x, err):
        x, err = x.reshape(-1), err.reshape(-1)
        if self.xbuf is None:
            self.xbuf = torch.empty((self.space, x.numel()), dtype=torch.float64, device=x.device)
            self.ebuf = torch.empty_like(self.xbuf)
            self.gram = torch.zeros((self.space, self.space), dtype=torch.float64, device=x.device)
        slot = self.count % self.space
        self.count += 1
        n = min(self.count, self.space)
        self.xbuf[slot].copy_(x)
        self.ebuf[slot].copy_(err)
        row = torch.mv(self.ebuf[:n], self.ebuf[slot])
        self.gram[slot, :n] = row
        self.gram[:n, slot] = row
        if n < 2:
            return x
        G = self.gram[:n, :n]
        B = torch.empty((n + 1, n + 1), dtype=torch.float64, device=x.device)
        B[:n, :n] = G / G.diagonal().abs().max().clamp_min(1e-300)
        B[n, :n] = B[:n, n] = -1.0
        B[n, n] = 0.0
        rhs = torch.zeros(n + 1, 1, dtype=torch.float64, device=x.device)
        rhs[n] = -1.0
        c = torch.linalg.lstsq(B, rhs).solution[:n, 0]
        return torch.mv(self.xbuf[:n].T, c)


_L_ERIS = ("fock", "mo_energy", "oooo", "ovoo", "ovvo", "oovv", "ovov", "ovvv", "vvvv")
_L_IMDS = ("w1", "w2", "w3", "w4", "woooo", "wvooo", "wVOov", "wvOOv", "wvvov")

MIXED_FLOOR = 1e-6     # update norm below which split-precision iterations stop helping


def kernel_gpu(mycc, eris=None, t1=None, t2=None, l1=None, l2=None, max_cycle=None, tol=None, verbose=None,
               use_cpu_vvvv=True, mode=None, polish=None):
    """Iterate to ||delta lambda|| < tol (ref: ccsd_gpu/gpu_ccsd_lambda.py:340-408).

    In a split-precision mode the iterations run in that mode down to
    max(tol, 1e-6); if ``tol`` is tighter and ``polish`` (default: the CC
    object's ``lambda_polish``, else True) is set, the intermediates are
    rebuilt in FP64 and FP64 iterations finish the solve (mixed-precision
    iterative refinement: the fixed point is the FP64 one).
    """
    _native.require_cuda()
    if eris is None:
        eris = mycc.ao2mo()
    eris = DeviceEris.wrap(eris)
    t1 = device_amp(mycc, "t1", mycc.t1 if t1 is None else t1)
    t2 = device_amp(mycc, "t2", mycc.t2 if t2 is None else t2)
    l1 = t1 if l1 is None else l1
    l2 = t2 if l2 is None else l2
    max_cycle = getattr(mycc, "max_cycle", 50) if max_cycle is None else max_cycle
    tol = getattr(mycc, "conv_tol_normt", 1e-5) if tol is None else tol
    mode = _mode_of(mycc, mode)
    polish = getattr(mycc, "lambda_polish", True) if polish is None else polish
    t1g, t2g, l1g, l2g = _t(t1), _t(t2), _t(l1), _t(l2)
    mode = effective_mode(mode, *t1g.shape)
    if t1g.data_ptr() == l1g.data_ptr() or t2g.data_ptr() == l2g.data_ptr():
        l1g, l2g = l1g.clone(), l2g.clone()
    mark_constant(t1g, t2g)
    cur_mode = mode
    cur_tol = tol if mode == "fp64" else max(tol, MIXED_FLOOR)
    imds = make_intermediates_gpu(mycc, t1g, t2g, eris, cur_mode)
    space = getattr(mycc, "diis_space", 6)
    use_diis = getattr(mycc, "diis", True)
    adiis = DIIS(space) if use_diis else None
    nov = l1g.numel()
    conv = False
    history = []
    graphs = getattr(mycc, "use_graphs", False)

    ls = float(getattr(mycc, "level_shift", 0.0))

    def make_step(im, md):
        if getattr(mycc, "use_graph_cache", True) and not graphs and graph_cache_ok(md, *t1g.shape):
            consts = {"e_" + k: getattr(eris, k) for k in _L_ERIS}
            consts.update({"i_" + k: getattr(im, k) for k in _L_IMDS})
            consts.update(t1=t1g, t2=t2g)
            key = ("L", t1g.shape[0], t1g.shape[1], ls, md)
            stub = SimpleNamespace(level_shift=ls)

            def body(c, a, b):
                er = SimpleNamespace(**{k: c["e_" + k] for k in _L_ERIS})
                imd = SimpleNamespace(mode=md, **{k: c["i_" + k] for k in _L_IMDS})
                return update_lambda_gpu(stub, c["t1"], c["t2"], a, b, er, imd, mode=md)
            return solve_step(key, body, consts)
        return StepGraph(lambda a, b: update_lambda_gpu(mycc, t1g, t2g, a, b, eris, im, mode=md), enabled=graphs)

    step = make_step(imds, cur_mode)
    for istep in range(max_cycle):
        l1n, l2n = step(l1g, l2g)
        normt = float(torch.sqrt(amplitude_norm_sq(l1n - l1g, l2n - l2g)))
        history.append((cur_mode, normt))
        if adiis is not None:
            x = torch.cat([l1n.reshape(-1), l2n.reshape(-1)])
            e = torch.cat([(l1n - l1g).reshape(-1), (l2n - l2g).reshape(-1)])
            x = adiis.update(x, e)
            l1n, l2n = x[:nov].reshape(l1g.shape), x[nov:].reshape(l2g.shape)
        l1g, l2g = l1n, l2n
        if normt < cur_tol:
            if cur_mode != "fp64" and polish and tol < cur_tol:
                cur_mode, cur_tol = "fp64", tol
                imds = make_intermediates_gpu(mycc, t1g, t2g, eris, "fp64")
                step = make_step(imds, cur_mode)
                adiis = DIIS(space) if use_diis else None
                continue
            # converged only if the requested tolerance was met: a split-precision
            # solve stopped at its noise floor without the FP64 polish is not
            conv = normt < tol
            break
    check_status()
    mycc._lambda_history = history
    # achieved update norm of the last iteration (the reference records only
    # the flag, ccsd_gpu/gpu_ccsd_lambda.py:445-448)
    mycc.lambda_normt = history[-1][1] if history else None
    mycc._last_lambda_dev = (l1g, l2g)
    return conv, host_copy(l1g), host_copy(l2g)


def solve_lambda_gpu(mycc, t1=None, t2=None, l1=None, l2=None, eris=None, use_cpu_vvvv=True,
                     fallback_to_cpu=True, mode=None):
    """Solve the Lambda equations; sets ``mycc.converged_lambda/l1/l2`` and
    ``mycc._lambda_solver_mode`` like the reference (ref: ccsd_gpu/gpu_ccsd_lambda.py:411-449)."""
    if not torch.cuda.is_available():
        raise RuntimeError("No usable CUDA device for the lambda solve (this package has no CPU path).")
    conv, l1o, l2o = kernel_gpu(mycc, eris=eris, t1=t1, t2=t2, l1=l1, l2=l2,
                                max_cycle=getattr(mycc, "max_cycle", 50),
                                tol=getattr(mycc, "conv_tol_normt", 1e-5), mode=mode)
    mycc.converged_lambda = conv
    mycc.l1 = l1o
    mycc.l2 = l2o
    l1g, l2g = mycc.__dict__.pop("_last_lambda_dev")
    remember_device(mycc, "l1", l1o, l1g)
    remember_device(mycc, "l2", l2o, l2g)
    mycc._lambda_solver_mode = "gpu-" + _mode_of(mycc, mode)
    return mycc.l1, mycc.l2
