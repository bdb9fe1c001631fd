"""Target-aware selection (SI_SEL_TARGET, opt-in) against the oracle.

The reference has no such mode (its selection is the same for every target,
pbwt_index.cpp:20-79); the oracle's restatement (oracle.select_pairs_target)
is pinned on the CPU against an explicit sort of reversed-prefix keys
(tests/test_oracle.py). Here the device walk gives the same slot pairs bit for
bit, and imputation with those per-target slots matches the FP64 oracle run on
each target with its own pairs: dosage and P(hap=1) within 1e-4, argmax
haplotypes bit-exact except where the oracle's own decision flips within
tie_eps +- 1e-5."""
import numpy as np
import pytest

import oracle
from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.fixture(scope="module")
def small():
    panel, _, _ = synth.make_panel(400, 300, 12, (0.3, 0.6), 0.01, 0.005, seed=5)
    codes, _, _ = synth.make_targets(panel, 24, synth.typed_every(400, 4), seed=6)
    codes[3, ::7] = 3                                    # a target with extra missing calls
    codes[5] = np.where(codes[5] == 1, 3, codes[5])      # one without heterozygous calls
    return panel, codes


def _setup(engine, panel, spacing):
    pos = (1 + np.arange(panel.shape[0], dtype=np.uint64) * np.uint64(spacing)).astype(np.uint64)
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build(store_index=True)
    return pos


@pytest.mark.parametrize("L", [4, 8, 16])
def test_target_pairs_bit_exact(engine, small, L):
    panel, codes = small
    _setup(engine, panel, 500_000)
    got = engine.select_states_target(L, codes)
    prefix = engine.prefix_rows()
    assert np.array_equal(prefix, oracle.pbwt_build(panel))
    for b in range(codes.shape[0]):
        want = oracle.select_pairs_target(prefix, panel, codes[b], L)
        assert np.array_equal(got[b], want), b
    # the slots follow the target: two targets differ somewhere
    assert not np.array_equal(got[0], got[1])


@pytest.mark.parametrize("spacing,L", [(500_000, 8), (1000, 8), (1000, 4)])
def test_target_imputation_against_oracle(engine, small, spacing, L):
    panel, codes = small
    pos = _setup(engine, panel, spacing)
    pairs = engine.select_states_target(L, codes)
    params = N.default_params(num_states=L, selection_kind=N.SEL_TARGET)
    out = engine.impute(codes, params, hap_prob=True)
    worst_d = worst_p = 0.0
    flips = 0
    for b in range(codes.shape[0]):
        want = oracle.fb_batch(codes[b:b + 1], pairs[b], panel, pos, L, float(params.ne))
        worst_d = max(worst_d, float(np.abs(out["dosage"][b] - want["dosage"][0]).max()))
        worst_p = max(worst_p, float(np.abs(out["hap_prob"][b] - want["hap_prob"][0]).max()))
        diff = out["haps"][b] != want["haps_argmax"][0]
        if diff.any():
            lo = oracle.fb_batch(codes[b:b + 1], pairs[b], panel, pos, L, float(params.ne), tie_eps=1e-4 - 1e-5)
            hi = oracle.fb_batch(codes[b:b + 1], pairs[b], panel, pos, L, float(params.ne), tie_eps=1e-4 + 1e-5)
            flip = (lo["haps_argmax"][0] != want["haps_argmax"][0]) | (hi["haps_argmax"][0] != want["haps_argmax"][0])
            assert not (diff & ~flip).any(), b
            flips += int(diff.sum())
    from conftest import report
    report(f"target-aware selection, {spacing} bp map, L={L}", targets=codes.shape[0],
           max_abs_dosage_diff=worst_d, max_abs_hap_prob_diff=worst_p, argmax_cells_differing=flips,
           cells=int(codes.size))
    assert worst_d <= TOL and worst_p <= TOL
    # the default (positional) selection is a different slot set, so the outputs differ
    default = engine.impute(codes, N.default_params(num_states=L))
    assert not np.array_equal(default["dosage"], out["dosage"])


def test_target_selection_refusals(engine, small):
    panel, codes = small
    pos = (1 + np.arange(panel.shape[0], dtype=np.uint64) * np.uint64(500_000)).astype(np.uint64)
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()  # head rows only
    params = N.default_params(num_states=8, selection_kind=N.SEL_TARGET)
    with pytest.raises(N.SIError, match="SI_PBWT_STORE_INDEX"):
        engine.impute(codes[:2], params)
    engine.pbwt_build(store_index=True)
    regions = [(0, 400, 8, N.INDEX_GLOBAL)]
    with pytest.raises(N.SIError, match="per target"):
        engine.impute_jobs(regions, [(0, codes[0], 0)], params)
