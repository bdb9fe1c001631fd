"""Plans (si_plan_*): a fixed uneven batch launched with no host work, plain
or as a captured CUDA graph, equals the uneven-batch entry point; the graph
replays on rewritten codes; the autotuner's choice stays within the tile bar;
a job beyond its anchor capacity is reported, not written out of bounds."""
import numpy as np
import pytest

from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth

pytestmark = pytest.mark.gpu


def _batch(engine, seed, n_jobs=40):
    panel, pos, _ = synth.make_panel(4000, 500, 16, seed=seed, spacing=100)
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()
    rng = np.random.default_rng(seed)
    regions = []
    for r in range(6):
        length = int(rng.integers(40, 1500))
        m0 = int(rng.integers(0, 4000 - length))
        regions.append((m0, m0 + length, [4, 8, 16][r % 3], [N.INDEX_REGION, N.INDEX_GLOBAL][r % 2]))

    def jobs_for(s):
        out = []
        for j in range(n_jobs):
            r = j % len(regions)
            m0, m1 = regions[r][:2]
            codes, _, _ = synth.make_targets(panel[m0:m1], 1, synth.typed_every(m1 - m0, 7), seed=s + j)
            out.append((r, codes[0], 1000 + j))
        return out
    return regions, jobs_for


def _equal(a, b, keys=("dosage", "haps")):
    for x, y in zip(a, b):
        for k in keys:
            assert np.array_equal(x[k], y[k]), k


@pytest.mark.parametrize("sampling", [N.SAMPLE_ARGMAX, N.SAMPLE_PHILOX])
def test_plan_and_graph_equal_jobs_path(engine, sampling):
    regions, jobs_for = _batch(engine, 31)
    params = N.default_params(sampling=sampling, seed=5)
    jobs = jobs_for(0)
    want = engine.impute_jobs(regions, jobs, params, hap_prob=True)
    plan = engine.plan(regions, jobs, params, hap_prob=True)
    try:
        plan.launch()
        _equal(plan.outputs(), want, ("dosage", "haps", "hap_prob"))
        plan.launch(graph=True)   # captures, then replays
        _equal(plan.outputs(), want, ("dosage", "haps", "hap_prob"))
        # new targets, same typed layout: rewrite the codes and replay the graph
        jobs2 = jobs_for(500)
        plan.set_codes([c for _, c, _ in jobs2])
        plan.launch(graph=True)
        _equal(plan.outputs(), engine.impute_jobs(regions, jobs2, params, hap_prob=True), ("dosage", "haps", "hap_prob"))
        assert plan.info()["window"] == 2
    finally:
        plan.destroy()


def test_autotuned_plan_within_tile_bar(engine):
    regions, jobs_for = _batch(engine, 32)
    jobs = jobs_for(0)
    want = engine.impute_jobs(regions, jobs, N.default_params())
    plan = engine.plan(regions, jobs, autotune=True)
    try:
        info = plan.info()
        assert info["window"] in (1, 2, 4) and info["threads"] in (32, 64, 128) and info["tuned_ms"] > 0
        plan.launch(graph=True)
        got = plan.outputs()
        for g, w in zip(got, want):
            assert np.abs(g["dosage"] - w["dosage"]).max() <= 2e-5
            assert np.array_equal(g["haps"], w["haps"])
    finally:
        plan.destroy()


def test_plan_capacity_overflow_is_reported(engine):
    regions, jobs_for = _batch(engine, 33, n_jobs=12)
    jobs = jobs_for(0)
    plan = engine.plan(regions, jobs, max_anchors=5)  # every job has more typed markers than that
    try:
        plan.launch(graph=True)
        with pytest.raises(N.SIError) as e:
            plan.check()
        assert e.value.status == 7  # SI_ERR_BUDGET
        plan.check()               # the flag was cleared
    finally:
        plan.destroy()
