"""Seeded SPD input generators.

Two groups:

* ``generate_input(batch, n, cond, seed, case)`` -- the reference task's six
  input families (reference/reference.py:37-126).  The random draws are made
  in the same order with the same torch calls, so on a given device they
  reproduce the reference's tensors exactly (pinned against the golden
  fixtures in ``tests/golden``).
* The five benchmark workloads: well-conditioned ``MM^T/n + I`` batches,
  prescribed-spectrum ``Q diag(lambda) Q^T`` batches, large ``GG^T/n + 0.1 I``
  matrices, a ragged list with log-uniform orders, and Gaussian-process RBF
  kernel matrices.  All are synthetic, seeded stand-ins.
"""

from __future__ import annotations

import math

import torch


def _sym(a: torch.Tensor) -> torch.Tensor:
    return 0.5 * (a + a.transpose(-1, -2))


def _orthogonal(batch: int, n: int, gen: torch.Generator, device) -> torch.Tensor:
    """Haar-like orthogonal factor: QR of a Gaussian matrix with R's diagonal signs folded in."""
    g = torch.randn((batch, n, n), device=device, dtype=torch.float32, generator=gen)
    q, r = torch.linalg.qr(g)
    sign = torch.where(
        torch.diagonal(r, dim1=-2, dim2=-1) >= 0, torch.ones((), device=device), -torch.ones((), device=device)
    )
    return q * sign.unsqueeze(-2)


def _gram_plus_diag(m: torch.Tensor, shift: float) -> torch.Tensor:
    """(M M^T)/n + shift*I, symmetrised."""
    n = m.shape[-1]
    g = (m @ m.transpose(-1, -2)) / float(max(n, 1))
    g.diagonal(dim1=-2, dim2=-1).add_(shift)
    return _sym(g).contiguous()


def generate_input(batch: int, n: int, cond: int, seed: int, case: str = "dense", device=None) -> torch.Tensor:
    """The reference task's input families (reference/reference.py:37-126).

    ``device`` defaults to CUDA when available, like the reference.
    """
    if batch <= 0 or n <= 0 or cond < 0:
        raise ValueError("batch and n must be positive and cond non-negative")
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    device = torch.device(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    case = case.lower()
    f32 = torch.float32
    if case == "dense":
        m = torch.randn((batch, n, n), device=device, dtype=f32, generator=gen)
        return _gram_plus_diag(m, 10.0 ** -max(cond, 2))
    if case == "diagonal":
        d = torch.logspace(0.0, -float(max(cond, 1)), n, device=device, dtype=f32)
        return torch.diag_embed(d.expand(batch, n)).contiguous()
    if case == "spectrum":
        lam = torch.logspace(0.0, -float(max(cond, 1)), n, device=device, dtype=f32).expand(batch, n)
        q = _orthogonal(batch, n, gen, device)
        return _sym((q * lam.unsqueeze(-2)) @ q.transpose(-1, -2)).contiguous()
    if case == "lowrank":
        rank = max(1, min(n // 8, 64))
        f = torch.randn((batch, n, rank), device=device, dtype=f32, generator=gen)
        g = (f @ f.transpose(-1, -2)) / float(rank)
        g.diagonal(dim1=-2, dim2=-1).add_(10.0 ** -max(cond, 3))
        return _sym(g).contiguous()
    if case == "rowscale":
        m = torch.randn((batch, n, n), device=device, dtype=f32, generator=gen)
        base = _gram_plus_diag(m, 1.0e-3)
        s = torch.logspace(0.0, -0.5 * float(max(cond, 2)), n, device=device, dtype=f32)
        g = s.reshape(1, n, 1) * base * s.reshape(1, 1, n)
        g.diagonal(dim1=-2, dim2=-1).add_(1.0e-6)
        return _sym(g).contiguous()
    if case == "tridiagonal":
        d = torch.empty((batch, n), device=device, dtype=f32).uniform_(1.5, 2.5, generator=gen)
        e = torch.empty((batch, max(n - 1, 0)), device=device, dtype=f32).uniform_(-0.25, 0.25, generator=gen)
        t = torch.diag_embed(d)
        if n > 1:
            t = t + torch.diag_embed(e, offset=1) + torch.diag_embed(e, offset=-1)
        return t.contiguous()
    raise ValueError(f"unknown Cholesky test case: {case}")


# ---------------------------------------------------------------------------
# Benchmark workloads (synthetic, seeded).


def well_conditioned(batch: int, n: int, seed: int, device="cpu") -> torch.Tensor:
    """A = (M M^T)/n + I, symmetrised, M ~ N(0,1) FP32."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    m = torch.randn((batch, n, n), device=device, dtype=torch.float32, generator=gen)
    return _gram_plus_diag(m, 1.0)


def prescribed_spectrum(batch: int, n: int, seed: int, lo: float = 1.0, hi: float = 1.0e6, device="cpu") -> torch.Tensor:
    """A = Q diag(lambda) Q^T, Q from QR of a Gaussian matrix, lambda log-spaced over [lo, hi]."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    lam = torch.logspace(math.log10(lo), math.log10(hi), n, device=device, dtype=torch.float32).expand(batch, n)
    q = _orthogonal(batch, n, gen, device)
    return _sym((q * lam.unsqueeze(-2)) @ q.transpose(-1, -2)).contiguous()


def mixed_batch(batch: int, n: int, seed: int, device="cpu") -> torch.Tensor:
    """First half well-conditioned, second half prescribed spectrum [1, 1e6]."""
    h = batch // 2
    a = well_conditioned(h, n, seed, device)
    b = prescribed_spectrum(batch - h, n, seed + 1, device=device)
    return torch.cat([a, b], dim=0).contiguous()


def large_gram(n: int, seed: int, device="cpu") -> torch.Tensor:
    """One matrix A = G G^T/n + 0.1 I, G ~ N(0,1) FP32, shape (1, n, n)."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    g = torch.randn((1, n, n), device=device, dtype=torch.float32, generator=gen)
    return _gram_plus_diag(g, 0.1)


def ragged_orders(count: int, seed: int, lo: int = 16, hi: int = 2048) -> list[int]:
    """n_i = round(exp(U[ln lo, ln hi])), seeded."""
    gen = torch.Generator(device="cpu")
    gen.manual_seed(seed)
    u = torch.rand(count, generator=gen, dtype=torch.float64)
    ln = math.log(lo) + u * (math.log(hi) - math.log(lo))
    return [int(round(math.exp(float(x)))) for x in ln]


def pack_offsets(orders: list[int]) -> list[int]:
    """Element offsets of a packed list; each matrix starts on a 16-byte boundary."""
    offs, pos = [], 0
    for n in orders:
        offs.append(pos)
        pos += ((n * n + 3) // 4) * 4
    offs.append(pos)
    return offs


def ragged_batch(orders: list[int], seed: int, device="cpu") -> tuple[torch.Tensor, list[int]]:
    """Packed buffer of M M^T/n + I matrices of the given orders; returns (buffer, offsets+[total])."""
    offs = pack_offsets(orders)
    buf = torch.zeros(offs[-1], dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    for i, n in enumerate(orders):
        m = torch.randn((1, n, n), device=device, dtype=torch.float32, generator=gen)
        buf[offs[i] : offs[i] + n * n] = _gram_plus_diag(m, 1.0).reshape(-1)
    return buf, offs


def rbf_kernel_batch(batch: int, n: int, seed: int, device="cpu") -> tuple[torch.Tensor, torch.Tensor]:
    """GP covariance: RBF over U[0,1]^3 points, lengthscale U[0.2,0.5], variance 1, +1e-4 I; y ~ N(0,1)."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    x = torch.rand((batch, n, 3), device=device, dtype=torch.float32, generator=gen)
    ls = 0.2 + 0.3 * torch.rand((batch, 1, 1), device=device, dtype=torch.float32, generator=gen)
    d2 = (x.unsqueeze(-2) - x.unsqueeze(-3)).pow(2).sum(-1)
    k = torch.exp(-0.5 * d2 / (ls * ls))
    k.diagonal(dim1=-2, dim2=-1).add_(1.0e-4)
    y = torch.randn((batch, n), device=device, dtype=torch.float32, generator=gen)
    return _sym(k).contiguous(), y
