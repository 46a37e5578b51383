"""Seeded synthetic Wigner coefficients for tests, the benchmark and the
serving trace.  The same buffer is fed to the GPU library and to the CPU
checker.  Distributions follow the workloads the transform path is measured
on: iid U(-1, 1) real and imaginary parts, or complex Gaussian with variance
proportional to (l+1)^-2; real signals satisfy f_{l,-m,0} = (-1)^m conj f_{l,m,0}
with real f_{l,0,0} (the reality condition of the reference's
tests/utilities.c:105-199).
"""
from __future__ import annotations

import numpy as np


def _plane_ns(p):
    N = p.N
    ns = list(range(0, N)) if p.reality else list(range(-N + 1, N))
    out = []
    for n in ns:
        if p.n_mode == 1 and n % 2:
            continue
        if p.n_mode == 2 and n % 2 == 0:
            continue
        if p.n_mode == 3 and abs(n) < N - 1:
            continue
        out.append(n)
    return out


def block_base(p, n: int) -> int:
    """Offset b such that (l, m, n) sits at b + l*l + l + m (reference
    src/c/so3_sampling.c:369-426 and :571-597)."""
    L, N = p.L, p.N
    compact = p.storage == 1

    def negfirst(n):
        if not compact:
            return (N - 1 + n) * L * L
        an = abs(n)
        off = (N - 1 + n) * L * L - (2 * N - 1) * (N - 1) * N // 6
        off += an * (2 * an + 1) * (an + 1) // 6 if n <= 0 else -(an * (2 * an - 1) * (an - 1) // 6)
        return off - n * n

    if p.reality:
        return negfirst(n) - negfirst(0)
    if p.n_order == 0:  # zero-first
        if not compact:
            return (-2 * n - 1 if n < 0 else 2 * n) * L * L
        an = abs(n)
        off = (2 * an - 1) * (3 * L * L - an * (an - 1)) // 3
        if n >= 0:
            off += L * L - n * n
        return off - n * n
    return negfirst(n)


def flmn_size(p) -> int:
    L, N = p.L, p.N
    if p.storage == 0:
        return N * L * L if p.reality else (2 * N - 1) * L * L
    return N * (6 * L * L - (N - 1) * (2 * N - 1)) // 6 if p.reality else (2 * N - 1) * (3 * L * L - N * (N - 1)) // 3


def gen_flmn(p, seed: int, dist: str = "uniform") -> np.ndarray:
    """Coefficients for l >= max(L0, |n|) in every n-block the n_mode allows."""
    rng = np.random.default_rng(seed)
    out = np.zeros(flmn_size(p), np.complex128)
    L = p.L
    for n in _plane_ns(p):
        lo = max(p.L0, abs(n))
        if p.n_mode == 4:  # only |n| = l
            if abs(n) < lo or abs(n) >= L:
                continue
            ls = np.array([abs(n)])
        else:
            ls = np.arange(lo, L)
        if ls.size == 0:
            continue
        e = np.concatenate([np.arange(l * l, l * l + 2 * l + 1) for l in ls])
        el = np.floor(np.sqrt(e)).astype(np.int64)
        cnt = e.size
        if dist == "uniform":
            v = rng.uniform(-1, 1, cnt) + 1j * rng.uniform(-1, 1, cnt)
        elif dist == "gauss":
            v = (rng.normal(size=cnt) + 1j * rng.normal(size=cnt)) / np.sqrt(2.0) / (el + 1.0)
        else:
            raise ValueError(dist)
        idx = block_base(p, n) + e
        if p.reality and n == 0:
            m = e - el * el - el
            v = np.where(m == 0, v.real + 0j, v)
            pos = m > 0
            # f_{l,-m,0} = (-1)^m conj f_{l,m,0}
            neg_idx = block_base(p, 0) + el[pos] * el[pos] + el[pos] - m[pos]
            out[idx] = v
            out[neg_idx] = np.where(m[pos] % 2, -1.0, 1.0) * np.conj(v[pos])
            continue
        out[idx] = v
    return out


def gen_flm(L: int, seed: int, dist: str = "gauss", mmax: int | None = None) -> np.ndarray:
    """S^2 coefficients flm (index l*l+l+m); |m| <= mmax only if given."""
    rng = np.random.default_rng(seed)
    e = np.arange(L * L)
    el = np.floor(np.sqrt(e)).astype(np.int64)
    m = e - el * el - el
    if dist == "gauss":
        v = (rng.normal(size=e.size) + 1j * rng.normal(size=e.size)) / np.sqrt(2.0) / (el + 1.0)
    else:
        v = rng.uniform(-1, 1, e.size) + 1j * rng.uniform(-1, 1, e.size)
    if mmax is not None:
        v = np.where(np.abs(m) <= mmax, v, 0)
    return v
