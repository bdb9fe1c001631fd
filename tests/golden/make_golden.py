#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference's own code.

  python tests/golden/make_golden.py cpu   PBWT prefix arrays from the reference's
                                           PBWTBuilder (oracle/_ref/libref_pbwt.so, CPU)
  python tests/golden/make_golden.py gpu [DIR]
                                           selection slots, log posteriors and argmax
                                           haplotypes from the reference's CUDA kernels
                                           (oracle/_ref/libref_gpu.so) on a B200; writes
                                           DIR/ref_gpu_kernels.npz (DIR defaults to tests/golden)

Both libraries are the reference compiled from its unmodified sources by
oracle/Makefile. Inputs come from the seeded synthetic generator, except the
8-haplotype x 10-marker panel, which is the reference repository's own
test_reference.vcf parsed as text (only when that tree is present).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from swiftimpute_b200 import synth  # noqa: E402

REF_TREE = oracle.REFERENCE_TREE


def parse_vcf_panel(path: Path) -> np.ndarray:
    rows = []
    for line in path.read_text().splitlines():
        if not line or line.startswith("#"):
            continue
        f = line.split("\t")
        alle = []
        for g in f[9:]:
            a, b = g.split(":")[0].replace("/", "|").split("|")
            alle += [int(a), int(b)]
        rows.append(alle)
    return np.array(rows, dtype=np.uint8)


def cpu():
    out = {}
    if (REF_TREE / "test_reference.vcf").exists():
        out["vcf_panel"] = parse_vcf_panel(REF_TREE / "test_reference.vcf")
    rng = np.random.default_rng(2024)
    out["rand_panel"] = (rng.random((200, 257)) < 0.3).astype(np.uint8)
    panel, _, _ = synth.make_panel(120, 4432, 40, seed=7)
    out["synth_panel"] = panel
    fix = {}
    for name, p in out.items():
        pre, div = oracle.ref_pbwt_build(p)
        assert np.array_equal(div, np.broadcast_to(np.arange(p.shape[0], dtype=np.uint32)[:, None], p.shape))
        fix[f"{name}"] = synth.pack_panel(p) if name == "synth_panel" else p
        fix[f"{name}_N"] = np.uint32(p.shape[1])
        if name == "synth_panel":
            # 4,432-haplotype rows: keep the row hashes and the selection-relevant head (first 128 entries)
            fix[f"{name}_prefix_head"] = pre[:, :128].astype(np.uint16)
            fix[f"{name}_row_hash"] = np.array([oracle.row_hash(r) for r in pre], dtype=np.uint64)
        else:
            fix[f"{name}_prefix"] = pre.astype(np.uint16)
    np.savez_compressed(HERE / "pbwt_reference_builder.npz", **fix)
    print("wrote", HERE / "pbwt_reference_builder.npz")


GPU_CASES = [
    # name, M, N, B, L, ne, spacing, typed_every
    ("uniform_L8", 300, 256, 6, 8, 10000, 500_000, 5),
    ("dense_L8", 300, 256, 6, 8, 10000, 100, 5),
    ("dense_L16_warp", 400, 200, 4, 16, 20000, 30, 4),
    ("dense_L16_bitonic", 60, 12000, 3, 16, 10000, 100, 3),
]


def gpu():
    fix = {}
    for i, (name, M, N, B, L, ne, spacing, every) in enumerate(GPU_CASES):
        panel, pos, _ = synth.make_panel(M, N, 12, seed=100 + i, spacing=spacing)
        codes, _, _ = synth.make_targets(panel, B, synth.typed_every(M, every), seed=99)
        gl = oracle.codes_to_gl(codes)
        slots, lp, haps, ms = oracle.ref_gpu_impute(panel, pos, gl, L, ne)
        fix[f"{name}_panel"] = synth.pack_panel(panel)
        fix[f"{name}_shape"] = np.array([M, N, B, L, ne, spacing, every], dtype=np.int64)
        fix[f"{name}_codes"] = codes
        fix[f"{name}_slots"] = slots
        fix[f"{name}_logpost"] = lp
        fix[f"{name}_haps"] = haps
        print(name, "stage ms", ms)
    out = Path(sys.argv[2] if len(sys.argv) > 2 else ROOT / "tests" / "golden") / "ref_gpu_kernels.npz"
    out.parent.mkdir(exist_ok=True)
    np.savez_compressed(out, **fix)
    print("wrote", out)


if __name__ == "__main__":
    {"cpu": cpu, "gpu": gpu}[sys.argv[1]]()
