"""Seeded synthetic inputs for the benchmarks and the full-size parity checks.

ERI microbenchmark shells: 4096 shells, l in {0, 1, 2} with probabilities
4/9, 3/9, 2/9, 1..6 primitives each, exponents log-uniform in [0.05, 1e4],
contraction coefficients uniform in [0.1, 1] then normalised with the PySCF
convention, centres uniform in a 12-bohr cube, every shell on its own centre.
"""
import numpy as np
import torch

from .gto.mole import BAS_SLOTS, PTR_ENV_START, normalized_coefficients


class ShellSet:
    """_atm/_bas/_env of a synthetic set of (decontracted) shells."""

    def __init__(self, atm, bas, env):
        self._atm = np.ascontiguousarray(atm, dtype=np.int32)
        self._bas = np.ascontiguousarray(bas, dtype=np.int32)
        self._env = np.ascontiguousarray(env, dtype=np.float64)

    @property
    def nbas(self):
        return len(self._bas)

    @property
    def lmax(self):
        return int(self._bas[:, 1].max())


def eri_bench_shells(nshell=4096, seed=0, lvals=(0, 1, 2), lprob=(4 / 9, 3 / 9, 2 / 9), max_prim=6,
                     box=12.0, exp_range=(0.05, 1e4)):
    rng = np.random.default_rng(seed)
    env = [0.0] * PTR_ENV_START
    atm, bas = [], []
    ls = rng.choice(np.asarray(lvals), size=nshell, p=np.asarray(lprob))
    for ish in range(nshell):
        xyz = rng.uniform(0.0, box, 3)
        ptr = len(env)
        env.extend(xyz.tolist())
        env.append(0.0)
        atm.append([1, ptr, 1, ptr + 3, 0, 0])
        l = int(ls[ish])
        nprim = int(rng.integers(1, max_prim + 1))
        es = np.sort(10.0 ** rng.uniform(np.log10(exp_range[0]), np.log10(exp_range[1]), nprim))[::-1]
        cs = rng.uniform(0.1, 1.0, nprim)
        cs = normalized_coefficients(l, es, cs[:, None])[:, 0]
        pe = len(env)
        env.extend(es.tolist())
        pc = len(env)
        env.extend(cs.tolist())
        bas.append([ish, l, nprim, 1, 0, pe, pc, 0])
    return ShellSet(np.array(atm).reshape(-1, 6), np.array(bas).reshape(-1, BAS_SLOTS), np.array(env))


def lclass(bas, q):
    """Unique L-class id of quartets q (n, 4): sorted (li>=lj), (lk>=ll), pair order."""
    l = bas[:, 1][q]
    a = np.maximum(l[:, 0], l[:, 1]) * 10 + np.minimum(l[:, 0], l[:, 1])
    b = np.maximum(l[:, 2], l[:, 3]) * 10 + np.minimum(l[:, 2], l[:, 3])
    return np.maximum(a, b) * 100 + np.minimum(a, b)


def candidate_quartets(nb, m, rng):
    """m uniformly drawn unique-order quartets (i>=j, k>=l, ij>=kl) of nb shells."""
    i = rng.integers(0, nb, m)
    j = rng.integers(0, nb, m)
    k = rng.integers(0, nb, m)
    l = rng.integers(0, nb, m)
    ij = np.stack([np.maximum(i, j), np.minimum(i, j)], 1)
    kl = np.stack([np.maximum(k, l), np.minimum(k, l)], 1)
    pij = ij[:, 0].astype(np.int64) * (ij[:, 0] + 1) // 2 + ij[:, 1]
    pkl = kl[:, 0].astype(np.int64) * (kl[:, 0] + 1) // 2 + kl[:, 1]
    swap = pkl > pij
    a = np.where(swap[:, None], kl, ij)
    b = np.where(swap[:, None], ij, kl)
    return np.concatenate([a, b], 1).astype(np.int32)


def first_candidate_chunk(shells, n, seed=1, oversample=4):
    """The first candidate chunk :func:`sample_quartets` draws for a sample of
    n: screening a prefix of it yields quartets that are a prefix, in draw
    order, of the same sample (a uniform subset of it)."""
    return candidate_quartets(shells.nbas, n * oversample + 1024, np.random.default_rng(seed))


def sample_quartets(shells, n, seed=1, schwarz_fn=None, threshold=1e-12, oversample=4):
    """Uniform sample of unique quartets (i>=j, k>=l, ij>=kl) passing the screen.

    schwarz_fn(pairs) -> Q for an (m, 2) array of shell pairs.  Quartets are
    returned sorted by L-class (the kernels process them class-batched).
    """
    rng = np.random.default_rng(seed)
    nb = shells.nbas
    out = []
    have = 0
    while have < n:
        m = (n - have) * oversample + 1024
        q = candidate_quartets(nb, m, rng)
        if schwarz_fn is not None:
            pairs = np.concatenate([q[:, :2], q[:, 2:]], 0)
            keys = pairs[:, 0].astype(np.int64) * nb + pairs[:, 1]
            uk, inv = np.unique(keys, return_inverse=True)
            vals = np.asarray(schwarz_fn(np.stack([uk // nb, uk % nb], 1).astype(np.int32)))
            qv = vals[inv]
            keep = qv[:m] * qv[m:] > threshold
            q = q[keep]
        out.append(q)
        have += len(q)
    q = np.concatenate(out, 0)[:n]
    order = np.argsort(lclass(shells._bas, q), kind="stable")
    return np.ascontiguousarray(q[order])


def ncart(l):
    return (l + 1) * (l + 2) // 2


def reference_flops(li, lj, lk, ll, npi, npj, npk, npl, deriv):
    """FP64 operation count of the reference algorithm for one shell quartet.

    Counted from the loop structure of fill_int2e_kernel / fill_int2e_ip1_kernel
    (ref: ccsd_gpu/cuda/int2e_module.py:253-430, ccsd_gpu/cuda/int2e_ip1_module.py:401-629),
    per primitive quartet: 29 for the Gaussian-product setup (:263-279), the
    Rys evaluation 2n (2*13 + 4) (ref: int2e_ip1_module.py:222-243), and per
    root 10 for the recurrence coefficients (:287-294), the vertical, transfer
    and two horizontal recurrences, and the accumulation (3 per output for
    int2e, 21 per output triple for int2e_ip1, ref: int2e_ip1_module.py:620-629).
    """
    nroots = (li + lj + lk + ll + deriv) // 2 + 1
    lij = li + lj + deriv
    lkl = lk + ll
    nf = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    sj = li + 1 + deriv
    sk = sj * (lj + 1)
    vrr = 3 * (1 + 4 * max(lij - 1, 0)) if lij > 0 else 0
    trr = 3 * (lij + 1) * lkl * 6
    hrr_ij = 3 * (lkl + 1) * sum(2 * (lij - j + 1) for j in range(lj))
    hrr_kl = 3 * sk * sum(2 * (lkl - l + 1) for l in range(ll))
    acc = (21 if deriv else 3) * nf
    per_root = 10 + vrr + trr + hrr_ij + hrr_kl + acc
    per_prim = 29 + 2 * nroots * (2 * 13 + 4) + nroots * per_root
    return per_prim * npi * npj * npk * npl


PAIR_CUT = 50.0     # primitive-pair screen of the ERI kernels (csrc/eri.cu kPairCut)


def kept_pairs(shells, i, j, extra_l=0, chunk=1 << 16):
    """Primitive pairs of the shell pairs (i[n], j[n]) that the ERI kernels
    keep: ab/(a+b) |AB|^2 <= PAIR_CUT + (li + lj + extra_l) ln(1 + |AB|)."""
    b, env, atm = shells._bas, shells._env, shells._atm
    i, j = np.asarray(i), np.asarray(j)
    mp = int(b[:, 2].max())
    E = np.full((len(b), mp), np.nan)
    for s in range(len(b)):
        E[s, :b[s, 2]] = env[b[s, 5]:b[s, 5] + b[s, 2]]
    R = np.stack([env[atm[b[s, 0], 1]:atm[b[s, 0], 1] + 3] for s in range(len(b))])
    out = np.empty(len(i), dtype=np.int64)
    for c0 in range(0, len(i), chunk):
        ii, jj = i[c0:c0 + chunk], j[c0:c0 + chunk]
        r2 = ((R[ii] - R[jj]) ** 2).sum(1)
        cut = PAIR_CUT + (b[ii, 1] + b[jj, 1] + extra_l) * np.log1p(np.sqrt(r2))
        ea, eb = E[ii][:, :, None], E[jj][:, None, :]
        with np.errstate(invalid="ignore"):
            th = ea * eb / (ea + eb) * r2[:, None, None]
            out[c0:c0 + chunk] = (th <= cut[:, None, None]).sum((1, 2))   # NaN (padding) compares False
    return out


def quartet_flops(shells, q, deriv, screened=True):
    """FP64 op count of the quartets q under the reference algorithm, over the
    primitive quartets that pass the kernels' pair screen (all of them with
    ``screened=False``)."""
    b = shells._bas
    l = b[:, 1][q]
    if screened:
        w = kept_pairs(shells, q[:, 0], q[:, 1], deriv) * kept_pairs(shells, q[:, 2], q[:, 3])
    else:
        w = b[:, 2][q].prod(1)
    total = 0
    keys, inv = np.unique(l, axis=0, return_inverse=True)
    wsum = np.bincount(inv.reshape(-1), weights=w.astype(np.float64), minlength=len(keys))
    for key, c in zip(keys, wsum):
        total += int(round(c)) * reference_flops(*[int(v) for v in key], 1, 1, 1, 1, deriv)
    return total


# ---- synthetic CCSD state for the Lambda / 2-RDM contraction benchmark ----------------
def _pair(a, b):
    hi, lo = torch.maximum(a, b), torch.minimum(a, b)
    return hi * (hi + 1) // 2 + lo


def synthetic_eri_block(z, P, Q, R, S, decay=0.1, out=None):
    """(pq|rs) over the index vectors P, Q, R, S of a symmetric random ERI tensor.

    (pq|rs) = z[canonical(p, q, r, s)] * exp(-decay * D) with the orbital
    distance D = |p-q| + |r-s| + (|p-r| + |q-s| + |p-s| + |q-r|) / 2: one random
    value per unique index quartet and a D that is invariant under the 8
    index permutations, so the tensor has the full 8-fold symmetry of real
    orbitals.  Evaluated slice by slice in P.
    """
    dev = z.device
    P, Q, R, S = (torch.as_tensor(x, dtype=torch.int64, device=dev) for x in (P, Q, R, S))
    pq = _pair(P[:, None], Q[None, :])
    rs = _pair(R[:, None], S[None, :])
    dpq = (P[:, None] - Q[None, :]).abs()
    drs = (R[:, None] - S[None, :]).abs()
    if out is None:
        out = torch.empty((len(P), len(Q), len(R), len(S)), dtype=torch.float64, device=dev)
    for p in range(len(P)):
        idx = _pair(pq[p][:, None, None], rs[None])
        a = (P[p] - R).abs()[None, :, None] + (Q[:, None, None] - S[None, None, :]).abs()
        b = (P[p] - S).abs()[None, None, :] + (Q[:, None, None] - R[None, :, None]).abs()
        dist = dpq[p][:, None, None] + drs[None] + 0.5 * (a + b)
        out[p] = z[idx] * torch.exp(-decay * dist.double())
    return out


def lambda_bench_state(nocc=24, nvir=216, seed=0, device="cuda", eri_sigma=0.05, decay=0.1):
    """Seeded synthetic CCSD state with PySCF's RCCSD integral layout.

    Orbital energies: sorted uniform in [-2, -0.3] Eh (occupied) and [0.1, 5] Eh
    (virtual); Fock matrix = diag(mo_energy).  t1 ~ N(0, 1e-3) and t2 ~ N(0,
    1e-2) (symmetrised to t2[ijab] = t2[jiba]), scaled by 1/(1 + |e_a - e_i|) and
    1/(1 + |e_a + e_b - e_i - e_j|).  MO ERIs: :func:`synthetic_eri_block` with
    values N(0, eri_sigma), decay constant 0.1 per orbital index step.  Returns
    (eris, t1, t2) with eris.{fock, mo_energy, oooo, ovoo, ovvo, oovv, ovov,
    ovvv, vvvv} as float64 tensors on ``device``.
    """
    from types import SimpleNamespace
    dev = torch.device(device)
    g = torch.Generator(device=dev).manual_seed(seed)
    nmo = nocc + nvir
    eo = torch.sort(torch.rand(nocc, generator=g, device=dev, dtype=torch.float64) * 1.7 - 2.0).values
    ev = torch.sort(torch.rand(nvir, generator=g, device=dev, dtype=torch.float64) * 4.9 + 0.1).values
    e = torch.cat([eo, ev])
    npair = nmo * (nmo + 1) // 2
    z = torch.randn(npair * (npair + 1) // 2, generator=g, device=dev, dtype=torch.float64) * eri_sigma
    o = torch.arange(nocc, device=dev)
    v = torch.arange(nocc, nmo, device=dev)
    blk = lambda a, b, c, d: synthetic_eri_block(z, a, b, c, d, decay)   # noqa: E731
    eris = SimpleNamespace(fock=torch.diag(e), mo_energy=e, oooo=blk(o, o, o, o), ovoo=blk(o, v, o, o),
                           ovvo=blk(o, v, v, o), oovv=blk(o, o, v, v), ovov=blk(o, v, o, v),
                           ovvv=blk(o, v, v, v), vvvv=blk(v, v, v, v))
    del z
    eia = eo[:, None] - ev[None, :]
    t1 = torch.randn(nocc, nvir, generator=g, device=dev, dtype=torch.float64) * 1e-3 / (1 + eia.abs())
    x = torch.randn(nocc, nocc, nvir, nvir, generator=g, device=dev, dtype=torch.float64)
    d2 = (eia[:, None, :, None] + eia[None, :, None, :]).abs()
    t2 = (x + x.permute(1, 0, 3, 2)) * (1e-2 / np.sqrt(2.0)) / (1 + d2)
    return eris, t1, t2


# ---- molecules of the gradient workloads ---------------------------------------------
def _zmat_to_xyz(rows):
    """Cartesian coordinates from (symbol, (i, r), (j, angle_deg), (k, dihedral_deg)) rows."""
    xyz = []
    for n, row in enumerate(rows):
        if n == 0:
            xyz.append(np.zeros(3))
            continue
        (i, r) = row[1]
        if n == 1:
            xyz.append(xyz[i] + np.array([r, 0.0, 0.0]))
            continue
        (j, ang) = row[2]
        a = np.radians(ang)
        if n == 2:
            u = (xyz[j] - xyz[i]) / np.linalg.norm(xyz[j] - xyz[i])
            v = np.array([-u[1], u[0], 0.0]) if abs(u[2]) < 0.9 else np.array([0.0, -u[2], u[1]])
            v /= np.linalg.norm(v)
            xyz.append(xyz[i] + r * (np.cos(a) * u + np.sin(a) * v))
            continue
        (k, dih) = row[3]
        d = np.radians(dih)
        b = xyz[i] - xyz[j]
        c = xyz[k] - xyz[j]
        nrm = np.cross(b, c)
        nrm /= np.linalg.norm(nrm)
        m = np.cross(nrm, b / np.linalg.norm(b))
        local = np.array([-r * np.cos(a), r * np.sin(a) * np.cos(d), r * np.sin(a) * np.sin(d)])
        bu = b / np.linalg.norm(b)
        xyz.append(xyz[i] + local[0] * bu + local[1] * m + local[2] * nrm)
    return np.array(xyz)


ETHANOL_ZMAT = [
    ("C",), ("C", (0, 1.512)), ("O", (1, 1.425), (0, 108.0)),
    ("H", (2, 0.962), (1, 108.5), (0, 180.0)),
    ("H", (1, 1.094), (2, 110.0), (3, 60.0)), ("H", (1, 1.094), (2, 110.0), (3, -60.0)),
    ("H", (0, 1.091), (1, 110.8), (2, 180.0)), ("H", (0, 1.091), (1, 110.8), (2, 60.0)),
    ("H", (0, 1.091), (1, 110.8), (2, -60.0)),
]


def ethanol_atoms(seed=0, sigma=0.02):
    """Ethanol (anti conformer) from standard bond lengths and angles
    (C-C 1.512, C-O 1.425, O-H 0.962, C-H 1.09 A; tetrahedral angles,
    staggered), displaced by seeded N(0, sigma A) noise: (symbols, xyz in A)."""
    xyz = _zmat_to_xyz(ETHANOL_ZMAT)
    xyz = xyz + np.random.default_rng(seed).normal(0.0, sigma, xyz.shape)
    return [r[0] for r in ETHANOL_ZMAT], xyz


_WATER = np.array([[0.0, 0.0, 0.0], [0.0, 0.757, 0.587], [0.0, -0.757, 0.587]])   # O, H, H (A)


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster_atoms(n, rng):
    """(H2O)n: each new oxygen 2.8 +- 0.2 A (uniform) from a randomly chosen
    earlier one and at least 2.5 A from all others, randomly oriented
    monomers with H atoms kept 1.5 A from other molecules' atoms."""
    mols = []
    for m in range(n):
        for _ in range(1000):
            R = _rotation(rng)
            if m == 0:
                centre = np.zeros(3)
            else:
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
                centre = mols[rng.integers(m)][0] + rng.uniform(2.6, 3.0) * d
            w = centre + _WATER @ R.T
            if all(np.linalg.norm(w[0] - o[0]) >= 2.5 for o in mols) and \
               all(np.linalg.norm(a - b) >= 1.5 for o in mols for a in w for b in o):
                mols.append(w)
                break
        else:
            raise RuntimeError("could not place water %d" % m)
    xyz = np.concatenate(mols, 0)
    return ["O", "H", "H"] * n, xyz


def water_clusters(count=64, seed=0, nmax=6):
    """`count` seeded clusters (H2O)n, n uniform in 1..nmax: list of (symbols, xyz A)."""
    rng = np.random.default_rng(seed)
    return [water_cluster_atoms(int(rng.integers(1, nmax + 1)), rng) for _ in range(count)]


def atom_string(symbols, xyz):
    return "; ".join("%s %.10f %.10f %.10f" % (s, *p) for s, p in zip(symbols, xyz))
