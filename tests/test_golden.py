"""The oracle against fixtures produced by the reference's own code
(tests/golden/make_golden.py): PBWT prefix arrays from its PBWTBuilder, and
selection / posteriors / argmax haplotypes from its CUDA kernels on a B200."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from swiftimpute_b200 import synth

GOLD = Path(__file__).resolve().parent / "golden"


def test_synth_pack_roundtrip():
    rng = np.random.default_rng(1)
    p = (rng.random((7, 91)) < 0.5).astype(np.uint8)
    assert np.array_equal(synth.unpack_panel(synth.pack_panel(p), 91), p)


def test_pbwt_reference_builder_goldens():
    g = np.load(GOLD / "pbwt_reference_builder.npz")
    names = [k for k in ("vcf_panel", "rand_panel") if k in g]
    assert "rand_panel" in names
    for name in names:
        assert np.array_equal(oracle.pbwt_build(g[name]), g[f"{name}_prefix"].astype(np.uint32))
    panel = synth.unpack_panel(g["synth_panel"], int(g["synth_panel_N"]))
    pre = oracle.pbwt_build(panel)
    assert np.array_equal(pre[:, :128], g["synth_panel_prefix_head"].astype(np.uint32))
    assert np.array_equal(np.array([oracle.row_hash(r) for r in pre], np.uint64), g["synth_panel_row_hash"])


def _ref_gpu():
    f = GOLD / "ref_gpu_kernels.npz"
    if not f.exists():
        pytest.skip("reference GPU fixtures not generated yet")
    return np.load(f)


CASES = ["uniform_L8", "dense_L8", "dense_L16_warp", "dense_L16_bitonic"]


def _case(g, name):
    M, N, B, L, ne, spacing, every = [int(x) for x in g[f"{name}_shape"]]
    panel = synth.unpack_panel(g[f"{name}_panel"], N)
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(spacing)).astype(np.uint64)
    return panel, pos, g[f"{name}_codes"], L, ne


@pytest.mark.parametrize("name", CASES)
def test_selection_matches_reference_kernels(name):
    g = _ref_gpu()
    panel, pos, codes, L, ne = _case(g, name)
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)
    assert np.array_equal(pairs[:, :, 0], g[f"{name}_slots"])


@pytest.mark.parametrize("name", CASES)
def test_posteriors_match_reference_kernels(name):
    """The reference's FP32 log-space kernels against the FP64 oracle: the
    posterior each samples from (softmax of its normalised log posterior).
    The reference's own FP32 rounding (unscaled beta near the e^-999 floor)
    measures up to ~1.2e-4 per probability on these cases (0 under the
    uniform map); the bar is 5e-4."""
    g = _ref_gpu()
    panel, pos, codes, L, ne = _case(g, name)
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)
    gl = oracle.codes_to_gl(codes)
    ref = g[f"{name}_logpost"].astype(np.float64)
    worst = 0.0
    for b in range(codes.shape[0]):
        lp = oracle.fb_logpost(gl[b], pairs, panel, pos, L, ne)
        P = np.exp(lp - lp.max(1, keepdims=True)); P /= P.sum(1, keepdims=True)
        R = np.exp(ref[b] - ref[b].max(1, keepdims=True)); R /= R.sum(1, keepdims=True)
        worst = max(worst, float(np.abs(P - R).max()))
    assert worst <= 5e-4, worst


def test_argmax_haplotypes_match_reference_under_exact_ties():
    """Under the 0.5 cM map every transition ties, so argmax ties are exact in
    both the reference's FP32 kernel and the oracle: haplotypes bit-exact."""
    g = _ref_gpu()
    panel, pos, codes, L, ne = _case(g, "uniform_L8")
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)
    want = oracle.fb_batch(codes, pairs, panel, pos, L, ne, tie_eps=0.0)
    assert np.array_equal(want["haps_argmax"], g["uniform_L8_haps"])
