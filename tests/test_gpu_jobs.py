"""Uneven batches: targets over different regions with different slot counts
in one launch sequence (si_impute_jobs_device), against the oracle run on the
corresponding panel slice, and each result identical alone and in the mix."""
import numpy as np
import pytest

import oracle
from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _setup(engine, M=2000, Nh=400, spacing=100, seed=50, irregular=False):
    panel, pos, _ = synth.make_panel(M, Nh, 16, seed=seed, spacing=spacing)
    if irregular:
        rng = np.random.default_rng(seed)
        pos = np.cumsum(rng.integers(20, 400, size=M)).astype(np.uint64)
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()
    return panel, pos


def _targets(panel, m0, m1, B, every, seed):
    typed = synth.typed_every(m1 - m0, every)
    codes, truth, _ = synth.make_targets(panel[m0:m1], B, typed, seed=seed)
    return codes


def _check(got, want, b):
    assert np.abs(got["dosage"] - want["dosage"][b]).max() <= TOL
    assert np.array_equal(got["haps"], want["haps_argmax"][b])


@pytest.mark.parametrize("origin", [N.INDEX_REGION, N.INDEX_GLOBAL])
def test_regions_against_oracle_on_slices(engine, origin):
    panel, pos = _setup(engine, irregular=(origin == N.INDEX_REGION))
    regions = [(0, 2000, 8, origin), (120, 700, 4, origin), (1500, 1960, 16, origin), (333, 334, 8, origin)]
    jobs, want = [], {}
    for r, (m0, m1, L, _) in enumerate(regions):
        codes = _targets(panel, m0, m1, 5, 4, seed=60 + r)
        sl = panel[m0:m1]
        if origin == N.INDEX_REGION:
            # the reference run on the sliced panel: sweep from the slice start, the slice's first gap
            pairs = oracle.select_pairs(oracle.pbwt_build(sl), L)
            spos = pos[m0:m1]
        else:
            # the resident index and the panel's first-gap matrix: give the oracle positions with that spacing
            pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)[m0:m1]
            d = int(pos[1] - pos[0])
            spos = (1 + np.arange(m1 - m0, dtype=np.uint64) * np.uint64(d)).astype(np.uint64)
        want[r] = oracle.fb_batch(codes, pairs, sl, spos, L, 10000.0)
        for b in range(codes.shape[0]):
            jobs.append((r, codes[b], 1000 * r + b))
    rng = np.random.default_rng(7)
    order = rng.permutation(len(jobs))
    shuffled = [jobs[i] for i in order]
    got = engine.impute_jobs(regions, shuffled, N.default_params(), hap_prob=True)
    for out, i in zip(got, order):
        r, _, sid = jobs[i]
        _check(out, want[r], sid - 1000 * r)


def test_job_alone_equals_job_in_the_mix(engine):
    panel, pos = _setup(engine, seed=51)
    regions = [(0, 1999, 16, N.INDEX_REGION), (10, 900, 8, N.INDEX_GLOBAL), (800, 1200, 4, N.INDEX_REGION)]
    jobs = []
    for r, (m0, m1, L, _) in enumerate(regions):
        codes = _targets(panel, m0, m1, 6, 5, seed=70 + r)
        jobs += [(r, codes[b], 10 * r + b) for b in range(6)]
    for sampling in (N.SAMPLE_ARGMAX, N.SAMPLE_PHILOX):
        p = N.default_params(sampling=sampling, seed=99)
        mix = engine.impute_jobs(regions, jobs, p, hap_prob=True)
        for i in (0, 7, 13, len(jobs) - 1):
            r = jobs[i][0]
            alone = engine.impute_jobs([regions[r]], [(0, jobs[i][1], jobs[i][2])], p, hap_prob=True)[0]
            for key in ("dosage", "haps", "hap_prob"):
                assert np.array_equal(alone[key], mix[i][key]), (i, key)


def test_haplotypes_without_dosage(engine):
    # argmax haplotypes alone (no dosage buffer: the posterior variant without the dosage sums)
    # equal those of the call that also writes dosage, for every job
    panel, pos = _setup(engine, seed=54)
    regions = [(0, 1999, 16, N.INDEX_REGION), (10, 900, 8, N.INDEX_GLOBAL), (800, 1200, 4, N.INDEX_REGION)]
    jobs = []
    for r, (m0, m1, L, _) in enumerate(regions):
        codes = _targets(panel, m0, m1, 5, 5, seed=90 + r)
        jobs += [(r, codes[b], 10 * r + b) for b in range(5)]
    p = N.default_params()
    both = engine.impute_jobs(regions, jobs, p)
    only = engine.impute_jobs(regions, jobs, p, dosage=False)
    for i in range(len(jobs)):
        assert "dosage" not in only[i]
        assert np.array_equal(only[i]["haps"], both[i]["haps"]), i


def test_plain_batch_equals_single_full_region(engine):
    panel, pos = _setup(engine, seed=52)
    codes = _targets(panel, 0, 2000, 8, 5, seed=80)
    plain = engine.impute(codes, N.default_params(), hap_prob=True)
    jobs = engine.impute_jobs([(0, 2000, 8, N.INDEX_GLOBAL)], [(0, codes[b], b) for b in range(8)],
                              N.default_params(), hap_prob=True)
    for b in range(8):
        assert np.array_equal(jobs[b]["dosage"], plain["dosage"][b])
        assert np.array_equal(jobs[b]["haps"], plain["haps"][b])


def test_bad_jobs_are_refused(engine):
    _setup(engine, seed=53)
    with pytest.raises(N.SIError):
        engine.impute_jobs([(5, 3, 8, N.INDEX_GLOBAL)], [(0, np.zeros(0, np.uint8), 0)])
    with pytest.raises(N.SIError):
        engine.impute_jobs([(0, 100, 40, N.INDEX_GLOBAL)], [(0, np.zeros(100, np.uint8), 0)])
