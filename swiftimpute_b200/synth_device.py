"""Seeded synthetic panels and targets generated on the device with torch.

The same recipe as swiftimpute_b200.synth (founder mosaic with allele flips;
targets a mosaic of panel haplotypes, typed at every k-th marker), for shapes
where a host generator would take minutes (a 100,000 x 100,000 byte panel is
10 GB). Targets are not resampled for heterozygosity. torch's device RNG makes
every draw reproducible from the seed on a given device type.
"""
from __future__ import annotations

import numpy as np


def make_panel(M: int, N: int, n_founders: int, beta=(0.5, 0.5), switch: float = 0.01, flip: float = 0.005,
               seed: int = 0, device="cuda", chunk: int = 2048):
    """u8 panel [M][N] on the device: founder alleles ~ Bernoulli(p_m), p_m ~ Beta(beta)."""
    import torch
    rng = np.random.default_rng(seed)
    p = rng.beta(beta[0], beta[1], size=M)
    fnd = torch.from_numpy((rng.random((n_founders, M)) < p[None, :]).astype(np.uint8)).to(device)
    g = torch.Generator(device=device).manual_seed(seed)
    panel = torch.empty((M, N), dtype=torch.uint8, device=device)
    carry = torch.randint(0, n_founders, (N,), generator=g, device=device)
    for m0 in range(0, M, chunk):
        c = min(M, m0 + chunk) - m0
        ar = torch.arange(c, device=device)[:, None]
        sw = torch.rand((c, N), generator=g, device=device) < switch
        new = torch.randint(0, n_founders, (c, N), generator=g, device=device)
        last = torch.cummax(torch.where(sw, ar, torch.full_like(ar, -1)).expand(c, N), dim=0).values
        idx = torch.where(last >= 0, torch.gather(new, 0, last.clamp(min=0)), carry[None, :])
        carry = idx[-1].clone()
        alle = fnd[idx, (m0 + ar).expand(c, N)]
        alle ^= (torch.rand((c, N), generator=g, device=device) < flip).to(torch.uint8)
        panel[m0:m0 + c] = alle
    return panel


def pack_panel(panel, chunk: int = 1024) -> np.ndarray:
    """Device u8 panel [M][N] (N a multiple of 32) -> host u32 [M][N/32], bit i of word w = haplotype 32 w + i."""
    import torch
    M, N = panel.shape
    W = N // 32
    shifts = torch.arange(32, device=panel.device, dtype=torch.int64)
    out = np.empty((M, W), dtype=np.uint32)
    for m0 in range(0, M, chunk):
        rows = panel[m0:m0 + chunk].view(-1, W, 32).to(torch.int64)
        words = (rows << shifts).sum(-1)  # distinct bits: the sum is the 32-bit word
        out[m0:m0 + chunk] = words.cpu().numpy().astype(np.uint32)
    return out


def make_targets(panel, B: int, every: int = 0, n_mosaic: int = 8, switch: float = 0.005, seed: int = 0,
                 chunk: int = 1024, typed=None):
    """Genotype codes [B][M] u8 on the device: h0 + h1 at the typed markers
    (m % every == 0, or the marker indices in ``typed``), 3 elsewhere."""
    import torch
    dev = panel.device
    M, N = panel.shape
    mask = torch.zeros(M, dtype=torch.bool, device=dev)
    if typed is not None:
        mask[torch.as_tensor(np.asarray(typed, dtype=np.int64), device=dev)] = True
    else:
        mask[::every] = True
    g = torch.Generator(device=dev).manual_seed(seed + 1000)
    H = 2 * B
    src = torch.randint(0, N, (H, n_mosaic), generator=g, device=dev)
    codes = torch.full((B, M), 3, dtype=torch.uint8, device=dev)
    carry = torch.randint(0, n_mosaic, (H,), generator=g, device=dev)
    for m0 in range(0, M, chunk):
        c = min(M, m0 + chunk) - m0
        ar = torch.arange(c, device=dev)[:, None]
        sw = torch.rand((c, H), generator=g, device=dev) < switch
        new = torch.randint(0, n_mosaic, (c, H), generator=g, device=dev)
        last = torch.cummax(torch.where(sw, ar, torch.full_like(ar, -1)).expand(c, H), dim=0).values
        k = torch.where(last >= 0, torch.gather(new, 0, last.clamp(min=0)), carry[None, :])
        carry = k[-1].clone()
        hap = torch.gather(src.t(), 0, k)                   # [c][H] panel haplotype per marker
        alle = torch.gather(panel[m0:m0 + c], 1, hap)       # [c][H]
        geno = alle[:, 0::2] + alle[:, 1::2]                # [c][B]
        typed = mask[m0:m0 + c, None].expand(c, B)
        codes[:, m0:m0 + c] = torch.where(typed, geno, torch.full_like(geno, 3)).t()
    return codes
