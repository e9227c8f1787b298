"""Seeded synthetic completion workloads with the shapes and value
distributions of the benchmark configurations (no public dataset is
available; these stand in for the reference's nell/DARPA/movielens/yelp
tensors).

Values: a rank-k CP model with N(0,1) factors, affinely mapped to [1, 5]
with the min/max over the generated cells, plus N(0, sigma^2) noise
(optionally clipped to [1, 5]).  Coordinates: uniform distinct cells, or
per-mode truncated Zipf(s) ranks mapped through a seeded permutation, with
duplicate cells removed and topped up until exactly nnz distinct cells
remain.  Train/test split by a seeded Bernoulli(train_frac).

Indices are returned 1-based (the .tns convention the reference needs).
Generation runs in torch on the given device (CUDA for the 100M-nonzero
workloads, CPU for small ones); the same seed on the same device type gives
the same tensor.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Workload:
    name: str
    dims: tuple
    nnz: int
    cp_rank: int
    rank: int
    sigma: float
    clip: bool
    zipf: tuple | None  # per-mode exponent, or None for uniform
    zipf_top: tuple | None = None  # per mode: expected nonzeros of the top row (Zipf-Mandelbrot offset), 0 = plain


WORKLOADS = {
    # 2,000 x 1,500 x 200, 200k uniform distinct cells, CP rank 8, R = 16
    "small-als": Workload("small-als", (2000, 1500, 200), 200_000, 8, 16, 0.1, False, None),
    # 500k x 20k x 2k, 100M Zipf(1.1) cells, CP rank 16, R = 32
    "zipf-100m": Workload("zipf-100m", (500_000, 20_000, 2_000), 100_000_000, 16, 32, 0.25, True,
                          (1.1, 1.1, 1.1)),
    # 400M Zipf(1.3) cells over 1M x 600k x 300, CP rank 24, R = 64.  I.i.d.
    # Zipf(1.3) in every mode puts about a quarter of the nonzeros in one
    # row of each large mode and cannot be deduplicated to 400M distinct
    # cells; the two large modes use a Zipf-Mandelbrot offset q, p(r) ~
    # (r + q)^-1.3, solved so that their top row holds 1e5 nonzeros (rows
    # then span 1 to ~1e5); the 300-row mode stays plain Zipf(1.3)
    "zipf-400m": Workload("zipf-400m", (1_000_000, 600_000, 300), 400_000_000, 24, 64, 0.2, False,
                          (1.3, 1.3, 1.3), (100_000, 100_000, 0)),
    # order 4: 250M Zipf(1.2) cells over 1M x 200k x 1k x 24, CP rank 32, R = 64
    "zipf4-250m": Workload("zipf4-250m", (1_000_000, 200_000, 1_000, 24), 250_000_000, 32, 64, 0.1, False,
                           (1.2, 1.2, 1.2, 1.2)),
}


def scaled(w: Workload, nnz: int, dims=None) -> Workload:
    """The same distribution with fewer nonzeros (and optionally other dims;
    the top-row targets scale with the nonzeros)."""
    top = None if w.zipf_top is None else tuple(int(t * nnz / w.nnz) for t in w.zipf_top)
    return Workload(w.name + f"@{nnz}", tuple(dims or w.dims), nnz, w.cp_rank, w.rank, w.sigma,
                    w.clip, w.zipf, top)


def zipf_offset(dim: int, s: float, n: int, top: float) -> float:
    """Offset q of the Zipf-Mandelbrot law p(r) ~ (r + q)^-s over ranks
    1..dim such that n * p(1) = top (bisection; 0 when plain Zipf already
    puts at most `top` nonzeros in the first rank)."""
    r = np.arange(1, dim + 1, dtype=np.float64)

    def first(q):
        w = (r + q) ** -s
        return n * w[0] / w.sum()

    if top <= 0 or first(0.0) <= top:
        return 0.0
    lo, hi = 0.0, float(dim)
    while first(hi) > top:
        hi *= 2.0
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if first(mid) > top:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _torch():
    import torch
    return torch


def _zipf_ranks(torch, n, dim, s, gen, device, q=0.0):
    # inverse CDF of the truncated Zipf(s) (offset q: Zipf-Mandelbrot) over
    # ranks 1..dim
    ranks = torch.arange(1, dim + 1, device=device, dtype=torch.float64)
    pmf = (ranks + q).pow(-s)
    cdf = torch.cumsum(pmf, 0)
    cdf = cdf / cdf[-1]
    u = torch.rand(n, generator=gen, device=device, dtype=torch.float64)
    return torch.searchsorted(cdf, u).clamp_(max=dim - 1)


def _draw_cells(torch, w: Workload, n, gen, device, perms):
    # mixed-radix cell keys (the product of the dimensions stays below 2^63)
    key = None
    for m, d in enumerate(w.dims):
        if w.zipf is None:
            c = torch.randint(0, d, (n,), generator=gen, device=device, dtype=torch.int64)
        else:
            q = zipf_offset(d, w.zipf[m], w.nnz, w.zipf_top[m]) if w.zipf_top else 0.0
            c = perms[m][_zipf_ranks(torch, n, d, w.zipf[m], gen, device, q)]
        key = c if key is None else key * d + c
    return key


def generate(w: Workload, seed: int = 0, device: str = "cpu", train_frac: float = 0.9):
    """Returns dict(train=(ind, vals), test=(ind, vals), dims) with numpy
    arrays (ind: 3 x n uint64 1-based, vals float64)."""
    torch = _torch()
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    perms = [torch.randperm(d, generator=gen, device=device) for d in w.dims]
    keys = torch.unique(_draw_cells(torch, w, w.nnz, gen, device, perms))
    tries = 0
    while keys.numel() < w.nnz and tries < 64:
        need = w.nnz - keys.numel()
        extra = _draw_cells(torch, w, int(need * 1.2) + 1024, gen, device, perms)
        keys = torch.unique(torch.cat([keys, extra]))
        tries += 1
    if keys.numel() < w.nnz:
        raise RuntimeError("could not draw enough distinct cells")
    # a seeded random subset of exactly nnz distinct cells
    sel = torch.randperm(keys.numel(), generator=gen, device=device)[: w.nnz]
    keys = keys[sel]
    cols = []
    for d in reversed(w.dims):
        cols.append(keys % d)
        keys = keys // d
    cols = cols[::-1]
    del keys, sel
    # values: rank-k CP model with N(0,1) factors
    F = [torch.randn(d, w.cp_rank, generator=gen, device=device, dtype=torch.float32) for d in w.dims]
    v = torch.empty(w.nnz, device=device, dtype=torch.float32)
    step = 1 << 24
    for s0 in range(0, w.nnz, step):
        sl = slice(s0, min(s0 + step, w.nnz))
        pr = F[0][cols[0][sl]]
        for m in range(1, len(w.dims)):
            pr = pr * F[m][cols[m][sl]]
        v[sl] = pr.sum(1)
        del pr
    lo, hi = v.min(), v.max()
    v = 1.0 + 4.0 * (v - lo) / (hi - lo)
    v = v.double() + w.sigma * torch.randn(w.nnz, generator=gen, device=device, dtype=torch.float64)
    if w.clip:
        v.clamp_(1.0, 5.0)
    train_mask = torch.rand(w.nnz, generator=gen, device=device) < train_frac
    ind = torch.stack(cols) + 1
    del cols

    def pack(mask):
        return (ind[:, mask].cpu().numpy().astype(np.uint64), v[mask].cpu().numpy())

    return dict(train=pack(train_mask), test=pack(~train_mask), dims=tuple(w.dims))


@dataclass
class BatchWorkload:
    name: str
    ninst: int
    dim_range: tuple   # each mode dimension log-uniform in [lo, hi]
    nnz_range: tuple   # nonzeros per instance log-uniform in [lo, hi]
    cp_rank: int
    rank: int
    sigma: float


BATCH_WORKLOADS = {
    # 256 instances, dims log-U[1e3, 5e4], nnz log-U[1e4, 5e6], uniform
    # distinct cells, CP rank 8 + N(0, 0.1^2), R = 16
    "batch-256": BatchWorkload("batch-256", 256, (1_000, 50_000), (10_000, 5_000_000), 8, 16, 0.1),
}


def batch_shapes(bw: BatchWorkload, seed: int = 0):
    """Per-instance (dims, nnz), drawn log-uniformly from a seeded numpy
    generator (the shapes do not depend on the device)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(bw.dim_range[0]), np.log(bw.dim_range[1])
    dims = np.exp(rng.uniform(lo, hi, (bw.ninst, 3))).astype(np.int64)
    lo, hi = np.log(bw.nnz_range[0]), np.log(bw.nnz_range[1])
    nnz = np.exp(rng.uniform(lo, hi, bw.ninst)).astype(np.int64)
    cells = dims.prod(axis=1)
    nnz = np.minimum(nnz, cells // 2)  # distinct cells stay drawable
    return [(tuple(int(x) for x in d), int(n)) for d, n in zip(dims, nnz)]


def generate_batch(bw: BatchWorkload, seed: int = 0, device: str = "cpu", train_frac: float = 0.9):
    """Yields one dict(train=(ind, vals), test=(ind, vals), dims) per
    instance: uniform distinct cells, values from the instance's own rank-k
    CP model mapped to [1, 5] plus N(0, sigma^2) noise (not clipped)."""
    for b, (dims, nnz) in enumerate(batch_shapes(bw, seed)):
        w = Workload(f"{bw.name}#{b}", dims, nnz, bw.cp_rank, bw.rank, bw.sigma, False, None)
        yield generate(w, seed=seed * 100_003 + b + 1, device=device, train_frac=train_frac)


def sort_for_mode(ind, vals, mode):
    """Stable sort by (ind[mode], ind[(mode+1)%3]) -- the reference's file order."""
    order = np.lexsort((ind[(mode + 1) % 3], ind[mode]))
    return ind[:, order], vals[order]


def random_small(nnz, dims, seed=0, low=1.0, high=5.0, distinct=True):
    """A small uniform test tensor (numpy only), 1-based indices."""
    rng = np.random.default_rng(seed)
    I, J, K = dims
    if distinct:
        total = I * J * K
        if nnz > total:
            raise ValueError("more nonzeros than cells")
        cells = rng.choice(total, size=nnz, replace=False)
        ind = np.stack([cells // (J * K), (cells // K) % J, cells % K]).astype(np.uint64) + 1
    else:
        ind = np.stack([rng.integers(0, d, nnz) for d in dims]).astype(np.uint64) + 1
    vals = rng.uniform(low, high, nnz)
    return ind, vals
