"""Serving loop (si_serve_*): requests queued from several threads and
batched continuously return exactly what each request returns imputed alone;
admission refuses what the launch size or the HBM budget cannot hold;
cancellation and statistics."""
import threading

import numpy as np
import pytest

from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth
from swiftimpute_b200.engine import Engine, Server

pytestmark = pytest.mark.gpu


def _setup(engine, M=3000, Nh=400, seed=90):
    panel, pos, _ = synth.make_panel(M, Nh, 16, seed=seed, spacing=100)
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()
    return panel


def _requests(panel, n, seed):
    rng = np.random.default_rng(seed)
    M = panel.shape[0]
    out = []
    for i in range(n):
        length = int(rng.integers(50, 900))
        m0 = int(rng.integers(0, M - length))
        L = int(rng.choice([4, 8, 16]))
        origin = int(rng.choice([N.INDEX_REGION, N.INDEX_GLOBAL]))
        B = int(rng.integers(1, 8))
        codes, _, _ = synth.make_targets(panel[m0:m0 + length], B, synth.typed_every(length, 5), seed=seed + i)
        out.append(dict(m0=m0, m1=m0 + length, L=L, origin=origin, codes=codes, sid=100 * i))
    return out


def _alone(engine, q, params):
    """The request imputed on its own through the uneven-batch entry point."""
    jobs = [(0, q["codes"][b], q["sid"] + b) for b in range(q["codes"].shape[0])]
    res = engine.impute_jobs([(q["m0"], q["m1"], q["L"], q["origin"])], jobs, params, hap_prob=True)
    return {"dosage": np.stack([r["dosage"] for r in res]), "haps": np.stack([r["haps"] for r in res]),
            "hap_prob": np.stack([r["hap_prob"] for r in res])}


def _same(got, want):
    for key in ("dosage", "haps", "hap_prob"):
        assert np.array_equal(got[key], want[key]), key


def _against_oracle(panel, reqs, got):
    """Served results (equal to the requests alone) against the FP64 oracle on
    each request's slice; the panel's map is uniform, so both index origins
    take the slice's own positions."""
    import oracle
    from conftest import r2_masked, report
    pos = 1 + np.arange(panel.shape[0], dtype=np.uint64) * np.uint64(100)
    full = {}
    dd = dp = 0.0
    gd, wd, cs = [], [], []
    for q, g in zip(reqs, got):
        sl = panel[q["m0"]:q["m1"]]
        if q["origin"] == N.INDEX_REGION:
            pairs = oracle.select_pairs(oracle.pbwt_build(sl), q["L"])
        else:
            if q["L"] not in full:
                full[q["L"]] = oracle.select_pairs(oracle.pbwt_build(panel), q["L"])
            pairs = full[q["L"]][q["m0"]:q["m1"]]
        want = oracle.fb_batch(q["codes"], pairs, sl, pos[q["m0"]:q["m1"]], q["L"], 10000.0)
        dd = max(dd, float(np.abs(g["dosage"] - want["dosage"]).max()))
        dp = max(dp, float(np.abs(g["hap_prob"] - want["hap_prob"]).max()))
        gd.append(g["dosage"].ravel()); wd.append(want["dosage"].ravel()); cs.append(q["codes"].ravel())
    r2 = r2_masked(np.concatenate(gd), np.concatenate(wd), np.concatenate(cs))
    report("serving requests, 24 mixed regions and L", targets=sum(q["codes"].shape[0] for q in reqs),
           max_abs_dosage_diff=dd, max_abs_hap_prob_diff=dp, dosage_r2_vs_oracle=r2)
    assert dd <= 1e-4 and dp <= 1e-4 and r2 >= 1 - 1e-6


@pytest.mark.parametrize("sampling", [N.SAMPLE_ARGMAX, N.SAMPLE_PHILOX])
def test_served_requests_equal_requests_alone(engine, sampling):
    panel = _setup(engine)
    params = N.default_params(sampling=sampling, seed=7)
    reqs = _requests(panel, 24, seed=300 + sampling)
    want = [_alone(engine, q, params) for q in reqs]
    with Server(engine, params, max_wait_us=2000) as srv:
        tickets = [None] * len(reqs)

        def submit(idx):
            for i in idx:
                q = reqs[i]
                tickets[i] = srv.submit(q["m0"], q["m1"], q["codes"], num_states=q["L"], index_origin=q["origin"],
                                        sample_id_base=q["sid"], hap_prob=True)

        threads = [threading.Thread(target=submit, args=(range(k, len(reqs), 3),)) for k in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for i, q in enumerate(reqs):
            _same(srv.wait(tickets[i], timeout_ms=60000), want[i])
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["cells"] == sum(q["codes"].size for q in reqs)
    if sampling == N.SAMPLE_ARGMAX:
        _against_oracle(panel, reqs, want)
    assert 1 <= st["batches"] < len(reqs)  # requests shared launches
    assert 0 < st["latency_p50_ms"] <= st["latency_p99_ms"] <= st["latency_max_ms"]


def test_request_alone_and_in_a_crowd(engine):
    panel = _setup(engine, seed=91)
    reqs = _requests(panel, 12, seed=400)
    with Server(engine, max_wait_us=100) as srv:
        q = reqs[0]
        alone = srv.wait(srv.submit(q["m0"], q["m1"], q["codes"], num_states=q["L"], index_origin=q["origin"],
                                    sample_id_base=q["sid"], hap_prob=True))
    with Server(engine, max_wait_us=5000) as srv:
        ts = [srv.submit(r["m0"], r["m1"], r["codes"], num_states=r["L"], index_origin=r["origin"],
                         sample_id_base=r["sid"], hap_prob=True) for r in reqs[1:6] + [q] + reqs[6:]]
        outs = [srv.wait(t) for t in ts]
        assert srv.stats()["batches"] < len(ts)
    _same(outs[5], alone)


def test_submit_refuses_what_would_fail_a_shared_launch(engine):
    """A region whose first two markers share a genetic position has no FP32
    first-gap transition. Its request is refused at submission, since in a
    launch it would fail the requests beside it; requests around it are served."""
    panel, pos, _ = synth.make_panel(600, 200, 8, seed=93, spacing=100)
    pos = pos.copy()
    pos[301:] -= np.uint64(100)  # markers 300 and 301 share a position
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()
    codes, _, _ = synth.make_targets(panel[300:400], 2, synth.typed_every(100, 5), seed=94)
    with Server(engine, max_wait_us=2000) as srv:
        with pytest.raises(N.SIError) as e:
            srv.submit(300, 400, codes, num_states=8, index_origin=N.INDEX_REGION)
        assert e.value.status == 4  # SI_ERR_UNSUPPORTED
        ok = [srv.submit(299, 399, codes, num_states=8, index_origin=N.INDEX_REGION),
              srv.submit(300, 400, codes, num_states=8, index_origin=N.INDEX_GLOBAL)]
        for t in ok:
            out = srv.wait(t)
            assert np.isfinite(out["dosage"]).all()
        st = srv.stats()
    assert st["completed"] == 2 and st["failed"] == 0


def test_admission_refuses_oversized_requests(engine):
    panel = _setup(engine, seed=92)
    q = _requests(panel, 1, seed=500)[0]
    with Server(engine, max_batch_cells=q["codes"].size - 1) as srv:
        with pytest.raises(N.SIError) as e:
            srv.submit(q["m0"], q["m1"], q["codes"], num_states=q["L"])
        assert e.value.status == 7  # SI_ERR_BUDGET
        M = panel.shape[0]
        with pytest.raises(N.SIError) as e:  # a slice that runs past the panel
            srv.submit(M - 10, M + 10, np.zeros((1, 20), np.uint8))
        assert e.value.status == 1  # SI_ERR_INVALID_ARG
        out = srv.wait(srv.submit(q["m0"], q["m1"], q["codes"][:1], num_states=q["L"]))
        assert out["dosage"].shape == (1, q["m1"] - q["m0"])


def test_hbm_budget_admission():
    # a context whose budget holds the panel, its index and small launches only
    eng = Engine(0)
    panel = _setup(eng, seed=93)
    used, _ = eng.memory()
    eng.close()
    eng = Engine(0, hbm_budget_bytes=used + (256 << 20))
    try:
        panel = _setup(eng, seed=93)
        rng = np.random.default_rng(5)
        # 3.9e6 cells fit one launch (2^22) but not the budget: L=16 scratch is ~86 B per cell at worst
        big = (rng.random((1300, 3000)) < 0.2).astype(np.uint8) * 3
        with Server(eng, max_batch_cells=1 << 22) as srv:
            with pytest.raises(N.SIError) as e:
                srv.submit(0, 3000, big, num_states=16, index_origin=N.INDEX_GLOBAL)
            assert e.value.status == 7
            q = _requests(panel, 1, seed=600)[0]
            out = srv.wait(srv.submit(q["m0"], q["m1"], q["codes"], num_states=q["L"], index_origin=q["origin"]))
            assert np.isfinite(out["dosage"]).all()
    finally:
        eng.close()


def test_cancel_queued_request(engine):
    panel = _setup(engine, seed=94)
    a, b = _requests(panel, 2, seed=700)
    with Server(engine, max_wait_us=1_500_000) as srv:
        ta = srv.submit(a["m0"], a["m1"], a["codes"], num_states=a["L"])
        tb = srv.submit(b["m0"], b["m1"], b["codes"], num_states=b["L"])
        assert srv.cancel(tb)           # still waiting for company
        assert not srv.cancel(tb)       # finished (cancelled) already
        with pytest.raises(N.SIError) as e:
            srv.wait(tb)
        assert e.value.status == 8      # SI_ERR_CANCELLED
        assert np.isfinite(srv.wait(ta)["dosage"]).all()
        st = srv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 1
