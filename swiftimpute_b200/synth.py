"""Seeded synthetic panels and targets with the shapes of the benchmark configs.

The reference's published run uses a cannabis amplicon dataset that is not
available; these generators stand in for it (and for every larger config)
with the stated shapes, allele-frequency distributions and mosaic structure:

* founders: allele frequency p_m ~ Beta(a, b) per marker, founder alleles ~ Bernoulli(p_m);
* panel haplotype: founder mosaic starting at a uniform founder, switching to a
  uniform founder with probability ``switch`` per marker, then each allele
  flipped with probability ``flip``;
* target haplotype: mosaic of ``n_mosaic`` distinct panel haplotypes with
  switch rate ``target_switch``; genotype = h0 + h1; samples are redrawn until
  the heterozygous fraction lies in ``het_range``;
* typed markers keep their genotype, all others are masked (code 3);
* positions pos_m = 1 + m * spacing (the reference reads no genetic map and
  uses pos / 1e8 Morgans, src/api/imputer.cpp:596-604).

numpy's PCG64 stream makes every draw reproducible from the seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

MISSING = 3


def _mosaic_paths(rng: np.random.Generator, H: int, m_count: int, switch: float, choices: int,
                  carry: np.ndarray | None) -> tuple[np.ndarray, np.ndarray]:
    """Source index in [0, choices) for H paths over m_count markers.

    At every marker a path switches with probability ``switch`` to a uniform
    choice (marker 0 of a fresh path always draws). Returns (idx [H][m], last).
    """
    sw = rng.random((H, m_count)) < switch
    if carry is None:
        sw[:, 0] = True
        carry = np.zeros(H, dtype=np.int64)
    new = rng.integers(0, choices, size=(H, m_count))
    cols = np.where(sw, np.arange(m_count)[None, :], -1)
    np.maximum.accumulate(cols, axis=1, out=cols)
    idx = np.where(cols >= 0, np.take_along_axis(new, np.maximum(cols, 0), axis=1), carry[:, None])
    return idx, idx[:, -1].copy()


def make_panel(M: int, N: int, n_founders: int, beta: tuple[float, float] = (0.5, 0.5), switch: float = 0.01,
               flip: float = 0.005, seed: int = 0, spacing: int = 500_000, chunk: int | None = None):
    """Return (panel u8 [M][N], pos u64 [M], founders u8 [F][M])."""
    rng = np.random.default_rng(seed)
    p = rng.beta(beta[0], beta[1], size=M)
    founders = (rng.random((n_founders, M)) < p[None, :]).astype(np.uint8)
    panel = np.empty((M, N), dtype=np.uint8)
    chunk = chunk or max(16, min(2048, (32 << 20) // max(N, 1)))
    carry = None
    for m0 in range(0, M, chunk):
        m1 = min(M, m0 + chunk)
        idx, carry = _mosaic_paths(rng, N, m1 - m0, switch, n_founders, carry)
        alle = founders[idx, np.arange(m0, m1)[None, :]]
        alle ^= (rng.random((N, m1 - m0)) < flip).astype(np.uint8)
        panel[m0:m1] = alle.T
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(spacing)).astype(np.uint64)
    return panel, pos, founders


def make_targets(panel: np.ndarray, B: int, typed: np.ndarray, n_mosaic: int = 8, switch: float = 0.005,
                 het_range: tuple[float, float] = (0.12, 0.40), seed: int = 0, max_tries: int = 20,
                 chunk: int = 1024):
    """Return (codes u8 [B][M] with 3 at masked markers, truth genotypes u8 [B][M], haps u8 [B][2][M])."""
    M, N = panel.shape
    rng = np.random.default_rng(seed)
    haps = np.empty((B, 2, M), dtype=np.uint8)
    todo = np.arange(B)
    for _ in range(max_tries):
        if todo.size == 0:
            break
        H = 2 * todo.size
        src = np.stack([rng.choice(N, size=n_mosaic, replace=False) for _ in range(H)])  # [H][n_mosaic]
        out = np.empty((H, M), dtype=np.uint8)
        carry = None
        for m0 in range(0, M, chunk):
            m1 = min(M, m0 + chunk)
            idx, carry = _mosaic_paths(rng, H, m1 - m0, switch, n_mosaic, carry)
            hap_id = np.take_along_axis(src, idx, axis=1)               # [H][cl]
            out[:, m0:m1] = panel[m0:m1][np.arange(m1 - m0)[None, :], hap_id]
        h = out.reshape(todo.size, 2, M)
        haps[todo] = h
        het = (h[:, 0] != h[:, 1]).mean(axis=1)
        ok = (het >= het_range[0]) & (het <= het_range[1])
        todo = todo[~ok]
    truth = haps[:, 0] + haps[:, 1]
    codes = np.full((B, M), MISSING, dtype=np.uint8)
    codes[:, typed] = truth[:, typed]
    return codes, truth.astype(np.uint8), haps


def typed_every(M: int, k: int) -> np.ndarray:
    return np.arange(0, M, k)


def typed_evenly(M: int, n: int) -> np.ndarray:
    return np.unique((np.arange(n, dtype=np.int64) * M) // n)


@dataclass
class Workload:
    name: str
    panel: np.ndarray
    pos: np.ndarray
    codes: np.ndarray
    truth: np.ndarray
    typed: np.ndarray
    L: int
    ne: int
    seed: int

    @property
    def imputed_cells(self) -> int:
        return int(self.codes.shape[0]) * int(self.codes.shape[1] - self.typed.size)


def plain_small(seed: int = 0, B: int = 444, M: int = 1644, N: int = 4432, spacing: int = 500_000) -> Workload:
    """Plain method, small: 4,432 x 1,644 panel, 40 founders, Beta(0.5, 0.5),
    switch 0.01, flip 0.005; 444 targets typed at every 5th marker; L=8, Ne=1e4."""
    panel, pos, _ = make_panel(M, N, 40, (0.5, 0.5), 0.01, 0.005, seed=seed, spacing=spacing)
    typed = typed_every(M, 5)
    codes, truth, _ = make_targets(panel, B, typed, seed=seed + 1000)
    return Workload("plain-small 4432x1644 B444 L8", panel, pos, codes, truth, typed, 8, 10000, seed)


def dense_cohort(seed: int = 1, B: int = 10_000, M: int = 50_000, N: int = 4432, n_typed: int = 3000,
                 spacing: int = 500_000) -> Workload:
    """Batched dense cohort: 4,432 x 50,000 panel, 100 founders; 10,000 targets
    typed at 3,000 evenly spaced markers; L=8, Ne=2e4."""
    panel, pos, _ = make_panel(M, N, 100, (0.5, 0.5), 0.01, 0.005, seed=seed, spacing=spacing)
    typed = typed_evenly(M, n_typed)
    codes, truth, _ = make_targets(panel, B, typed, seed=seed + 1000)
    return Workload(f"dense-cohort {N}x{M} B{B} typed{n_typed} L8", panel, pos, codes, truth, typed, 8, 20000, seed)


def pack_panel(panel: np.ndarray) -> np.ndarray:
    """u8 [M][N] (0/1) -> u32 [M][ceil(N/32)], bit i of word w = haplotype 32w+i."""
    M, N = panel.shape
    W = (N + 31) // 32
    padded = np.zeros((M, W * 32), dtype=np.uint8)
    padded[:, :N] = panel
    bits = np.packbits(padded.reshape(M, W, 4, 8)[:, :, :, ::-1], axis=-1).reshape(M, W, 4)
    return (bits[..., 0].astype(np.uint32) | (bits[..., 1].astype(np.uint32) << 8)
            | (bits[..., 2].astype(np.uint32) << 16) | (bits[..., 3].astype(np.uint32) << 24))


def unpack_panel(words: np.ndarray, N: int) -> np.ndarray:
    """Inverse of pack_panel: u32 [M][W] -> u8 [M][N]."""
    words = np.ascontiguousarray(words, dtype=np.uint32)
    M, W = words.shape
    b = words.view(np.uint8).reshape(M, W, 4)
    bits = np.unpackbits(b, axis=-1, bitorder="little").reshape(M, W * 32)
    return bits[:, :N].astype(np.uint8)
