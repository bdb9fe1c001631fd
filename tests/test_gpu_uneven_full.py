"""The uneven-batch workload at full shape: an 8,000 x 120,000 panel, 64
regions of 500-20,000 markers (log-uniform length, uniform start), 4,096
targets spread uniformly over the regions, L in {4, 8, 16} per region, typed
every 5th marker, each region indexed from its own first marker (the
reference's sliced-panel run).

Checked at full size through properties (finite outputs in range, haplotype
alleles 0/1, jobs re-run alone bit-equal) and, every target, against the FP64
oracle (about 2.2e7 cells, seconds on the host's threads), on the 0.5 cM map
and on a 1 kb map."""
import numpy as np
import pytest

import oracle
from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.fixture(scope="module")
def workload(engine):
    rng = np.random.default_rng(2)
    M, Nh = 120_000, 8000
    panel, pos, _ = synth.make_panel(M, Nh, 200, (0.3, 0.6), 0.002, 0.005, seed=2)
    regions = []
    for _ in range(64):
        length = int(np.exp(rng.uniform(np.log(500), np.log(20_000))))
        m0 = int(rng.integers(0, M - length))
        regions.append((m0, m0 + length, int(rng.choice([4, 8, 16])), N.INDEX_REGION))
    assign = rng.integers(0, 64, size=4096)
    codes = {}
    for r, (m0, m1, _, _) in enumerate(regions):
        n = int((assign == r).sum())
        if n:
            codes[r], _, _ = synth.make_targets(panel[m0:m1], n, synth.typed_every(m1 - m0, 5), seed=100 + r)
    jobs, seen = [], {r: 0 for r in codes}
    for j, r in enumerate(assign):
        r = int(r)
        jobs.append((r, codes[r][seen[r]], j))
        seen[r] += 1
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()
    out = engine.impute_jobs(regions, jobs, N.default_params(), hap_prob=True)
    return panel, pos, regions, jobs, out


def test_full_shape_properties(workload):
    _, _, regions, jobs, out = workload
    cells = 0
    for (r, c, _), o in zip(jobs, out):
        n = regions[r][1] - regions[r][0]
        assert o["dosage"].shape == (n,) and o["haps"].shape == (2, n)
        assert np.isfinite(o["dosage"]).all() and (o["dosage"] >= -1e-6).all() and (o["dosage"] <= 2 + 1e-5).all()
        assert np.isin(o["haps"], (0, 1)).all()
        cells += n
    assert len(out) == 4096 and 1.5e7 < cells < 4e7


def test_full_shape_jobs_alone_equal_mix(engine, workload):
    _, _, regions, jobs, out = workload
    for j in np.random.default_rng(9).choice(len(jobs), 6, replace=False):
        r, c, sid = jobs[j]
        alone = engine.impute_jobs([regions[r]], [(0, c, sid)], N.default_params(), hap_prob=True)[0]
        for key in ("dosage", "haps", "hap_prob"):
            assert np.array_equal(alone[key], out[j][key]), (int(j), key)


def _check_all_against_oracle(panel, pos, regions, jobs, out, name):
    """Every target against the FP64 oracle on its region's own slice, index and transition."""
    worst_d = worst_p = 0.0
    flips = 0
    gots, wants, masks = [], [], []
    for r, (m0, m1, L, _) in enumerate(regions):
        idx = [j for j, (rr, _, _) in enumerate(jobs) if rr == r]
        if not idx:
            continue
        sl = panel[m0:m1]
        pairs = oracle.select_pairs(oracle.pbwt_build(sl), L)
        codes = np.stack([jobs[j][1] for j in idx])
        want = oracle.fb_batch(codes, pairs, sl, pos[m0:m1], L, 10000.0)
        for b, j in enumerate(idx):
            worst_d = max(worst_d, float(np.abs(out[j]["dosage"] - want["dosage"][b]).max()))
            worst_p = max(worst_p, float(np.abs(out[j]["hap_prob"] - want["hap_prob"][b]).max()))
            gots.append(out[j]["dosage"])
            wants.append(want["dosage"][b])
            masks.append(codes[b])
            diff = out[j]["haps"] != want["haps_argmax"][b]
            if diff.any():
                lo = oracle.fb_batch(codes[b:b + 1], pairs, sl, pos[m0:m1], L, 10000.0, tie_eps=1e-4 - 1e-5)
                hi = oracle.fb_batch(codes[b:b + 1], pairs, sl, pos[m0:m1], L, 10000.0, tie_eps=1e-4 + 1e-5)
                flip = (lo["haps_argmax"][0] != want["haps_argmax"][b]) | (hi["haps_argmax"][0] != want["haps_argmax"][b])
                assert not (diff & ~flip).any(), (name, j)
                flips += int(diff.sum())
    from conftest import r2_masked, report
    r2 = r2_masked(np.concatenate(gots), np.concatenate(wants), np.concatenate(masks))
    report(name, targets=len(gots), max_abs_dosage_diff=worst_d, max_abs_hap_prob_diff=worst_p,
           dosage_r2_vs_oracle=r2, argmax_cells_differing=flips, cells=int(sum(g.size for g in gots)))
    assert worst_d <= TOL and worst_p <= TOL
    assert r2 >= 1 - 1e-6
    assert len(gots) == len(jobs)


def test_full_shape_every_target_against_oracle(workload):
    panel, pos, regions, jobs, out = workload
    _check_all_against_oracle(panel, pos, regions, jobs, out, "uneven full shape, 0.5 cM map, every target")


def test_full_shape_dense_map_every_target_against_oracle(engine, workload):
    # markers 1 kb apart: each region's first-gap transition keeps memory (rho < 1)
    panel, _, regions, jobs, _ = workload
    pos = (1 + np.arange(panel.shape[0], dtype=np.uint64) * np.uint64(1000)).astype(np.uint64)
    engine.set_map(pos)
    out = engine.impute_jobs(regions, jobs, N.default_params(), hap_prob=True)
    _check_all_against_oracle(panel, pos, regions, jobs, out, "uneven full shape, 1 kb map, every target")
