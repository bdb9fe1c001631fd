"""Device kernels against the CPU oracle, through the C ABI (B200 only).

Bars: PBWT prefix rows, row hashes and selected pairs are bit-exact;
posterior dosage and P(hap=1) within 1e-4 absolute of the FP64 oracle; argmax
haplotypes bit-exact except at cells where the oracle's own decision flips
when the tie threshold moves by 1e-5 relative (there a slot's posterior sits
within FP32 round-off of the threshold); Philox-sampled haplotypes equal
except at draws within FP32 rounding of a slot boundary (<= 1e-3 of cells).
"""
import numpy as np
import pytest

import oracle
from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth

pytestmark = pytest.mark.gpu

DOSAGE_TOL = 1e-4


def load(engine, panel, pos, store=True):
    engine.upload_panel(panel)
    engine.set_map(pos)
    return engine.pbwt_build(store_index=store, row_hashes=True)


# ----------------------------------------------------------------------------- PBWT

@pytest.mark.parametrize("M,N_,p1", [(1, 2, 0.5), (10, 8, 0.5), (300, 333, 0.3), (1644, 4432, 0.2),
                                     (37, 32, 0.5), (64, 40000, 0.25)])
def test_pbwt_prefix_bit_exact(engine, M, N_, p1):
    rng = np.random.default_rng(M * 7 + N_)
    panel = (rng.random((M, N_)) < p1).astype(np.uint8)
    load(engine, panel, 1 + np.arange(M, dtype=np.uint64) * 100)
    want = oracle.pbwt_build(panel)
    got = engine.prefix_rows()
    assert np.array_equal(got, want)
    assert np.array_equal(engine.row_hashes(), oracle.pbwt_build_packed(synth.pack_panel(panel), N_)[1])


def test_pbwt_packed_upload_equals_u8(engine):
    rng = np.random.default_rng(3)
    panel = (rng.random((200, 1000)) < 0.4).astype(np.uint8)
    engine.upload_packed(synth.pack_panel(panel), 1000)
    engine.set_map(1 + np.arange(200, dtype=np.uint64))
    engine.pbwt_build(store_index=True)
    assert np.array_equal(engine.prefix_rows(), oracle.pbwt_build(panel))


def with_other_alleles(panel, seed, missing=0.01, multi=0.004):
    """A panel as a VCF with '.' calls and multi-allelic sites loads it: ALLELE_MISSING (255) and allele 2."""
    rng = np.random.default_rng(seed)
    out = panel.copy()
    u = rng.random(out.shape)
    out[u < missing] = 255
    out[(u >= missing) & (u < missing + multi)] = 2
    return out


def test_pbwt_with_missing_and_multiallelic_alleles(engine):
    # every non-zero byte goes to the "1" side (pbwt_index.cpp:183)
    rng = np.random.default_rng(60)
    panel = with_other_alleles((rng.random((400, 2000)) < 0.3).astype(np.uint8), 61)
    load(engine, panel, 1 + np.arange(400, dtype=np.uint64) * 100)
    assert engine.exception_count() == int((panel > 1).sum())
    assert np.array_equal(engine.prefix_rows(), oracle.pbwt_build(panel))
    assert np.array_equal(engine.row_hashes(), oracle.pbwt_build_packed(synth.pack_panel(panel != 0), 2000)[1])


# ----------------------------------------------------------------------------- selection

@pytest.mark.parametrize("N_,L,kind", [(4432, 8, N.SEL_AUTO), (300, 16, N.SEL_WARP), (300, 16, N.SEL_INSERTION),
                                       (12000, 16, N.SEL_AUTO), (40, 6, N.SEL_WARP), (5, 8, N.SEL_INSERTION),
                                       (4432, 48, N.SEL_AUTO), (4432, 1, N.SEL_AUTO)])
def test_selection_bit_exact(engine, N_, L, kind):
    rng = np.random.default_rng(N_ + L)
    panel = (rng.random((90, N_)) < 0.3).astype(np.uint8)
    load(engine, panel, 1 + np.arange(90, dtype=np.uint64), store=False)
    got = engine.select_states(L, kind)
    want = oracle.select_pairs(oracle.pbwt_build(panel), L, kind)
    assert np.array_equal(got, want)
    assert np.array_equal(engine.select_states(L, kind, 10, 20), want[10:20])


# ----------------------------------------------------------------------------- forward-backward

def workload(M, N_, B, typed, spacing, seed, founders=20, switch=0.01):
    panel, pos, _ = synth.make_panel(M, N_, founders, seed=seed, spacing=spacing, switch=switch)
    codes, truth, _ = synth.make_targets(panel, B, typed, seed=seed + 1)
    return panel, pos, codes, truth


def compare(engine, panel, pos, codes, L, ne, per_gap=False, sampling=N.SAMPLE_ARGMAX, seed=12345, sid=0,
            **kw):
    load(engine, panel, pos, store=False)
    p = N.default_params(num_states=L, ne=ne, transition_mode=N.TRANS_PER_GAP if per_gap else N.TRANS_MATRIX0,
                         sampling=sampling, seed=seed, sample_id_base=sid, **kw)
    got = engine.impute(codes, p, hap_prob=True)
    pairs = engine.select_states(L)
    assert np.array_equal(pairs, oracle.select_pairs(oracle.pbwt_build(panel), L))
    want = oracle.fb_batch(codes, pairs, panel, pos, L, ne, per_gap=per_gap, tie_eps=p.tie_eps, seed=seed,
                           sample_id_base=sid, sampled=sampling == N.SAMPLE_PHILOX)
    dd = np.abs(got["dosage"] - want["dosage"]).max()
    dp = np.abs(got["hap_prob"] - want["hap_prob"]).max()
    assert dd <= DOSAGE_TOL, f"max |d dosage| = {dd}"
    assert dp <= DOSAGE_TOL, f"max |d P(hap=1)| = {dp}"
    if sampling == N.SAMPLE_ARGMAX:
        diff = (got["haps"] != want["haps_argmax"]).any(axis=1)
        if diff.any():
            lo = oracle.fb_batch(codes, pairs, panel, pos, L, ne, per_gap=per_gap, tie_eps=p.tie_eps - 1e-5)
            hi = oracle.fb_batch(codes, pairs, panel, pos, L, ne, per_gap=per_gap, tie_eps=p.tie_eps + 1e-5)
            flip = ((lo["haps_argmax"] != want["haps_argmax"]) | (hi["haps_argmax"] != want["haps_argmax"])).any(axis=1)
            assert not (diff & ~flip).any(), f"{int((diff & ~flip).sum())} argmax cells differ away from the threshold"
    else:
        frac = np.mean(got["haps"] != want["haps_sampled"])
        assert frac <= 1e-3, f"sampled haplotypes differ at {frac:.2e} of cells"
    return got, want


@pytest.mark.parametrize("spacing", [500_000, 1000, 100])
def test_fb_plain_small_shape(engine, spacing):
    # the plain-method config (4,432 haplotypes x 1,644 markers, every 5th typed, L=8, Ne=1e4), all 444
    # targets, on the 0.5 cM map (memoryless: rho clamps to 1) and on 1 kb and 100 bp maps
    panel, pos, codes, _ = workload(1644, 4432, 444, synth.typed_every(1644, 5), spacing, 0, founders=40)
    got, want = compare(engine, panel, pos, codes, 8, 10000)
    from conftest import r2_masked, report
    r2 = r2_masked(got["dosage"], want["dosage"], codes)
    report(f"plain-small spacing {spacing}", targets=444, max_abs_dosage_diff=np.abs(got["dosage"] - want["dosage"]).max(),
           max_abs_hap_prob_diff=np.abs(got["hap_prob"] - want["hap_prob"]).max(), dosage_r2_vs_oracle=r2,
           argmax_cells_differing=int((got["haps"] != want["haps_argmax"]).sum()))
    assert r2 >= 1 - 1e-6


@pytest.mark.parametrize("L", [1, 2, 3, 4, 5, 8, 13, 16, 24, 32])
def test_fb_state_counts(engine, L):
    panel, pos, codes, _ = workload(777, 600, 70, synth.typed_every(777, 4), 150, 5)
    compare(engine, panel, pos, codes, L, 10000)


def test_fb_per_gap_irregular_map(engine):
    panel, _, codes, _ = workload(500, 700, 33, synth.typed_every(500, 3), 100, 7)
    rng = np.random.default_rng(8)
    pos = np.cumsum(rng.integers(1, 3000, size=500)).astype(np.uint64)
    compare(engine, panel, pos, codes, 8, 10000, per_gap=True)
    compare(engine, panel, pos, codes, 8, 10000, per_gap=False)


def test_fb_floor_regime(engine):
    # long untyped runs under the uniform map drive beta to the e^-999 floor
    panel, pos, codes, _ = workload(2000, 300, 40, np.array([0, 10, 700, 1999]), 500_000, 9)
    compare(engine, panel, pos, codes, 8, 10000)
    panel, pos, codes, _ = workload(3000, 300, 40, np.array([0, 5, 2990]), 30, 10)
    compare(engine, panel, pos, codes, 16, 20000)


@pytest.mark.parametrize("L,flags", [(8, 0), (16, 0), (8, N.IMPUTE_FULL_CHAIN)])
def test_fb_panel_with_missing_and_multiallelic_alleles(engine, L, flags):
    # emission classes by the pair's byte sum (emission.cu:35-54), argmax
    # haplotypes carry the panel byte (sampling.cu:121-126); dosage and
    # P(hap=1) count non-zero alleles
    panel, pos, codes, _ = workload(900, 700, 48, synth.typed_every(900, 4), 100, 62)
    panel = with_other_alleles(panel, 63)
    got, want = compare(engine, panel, pos, codes, L, 10000, flags=flags)
    assert np.isin(got["haps"], [2, 255]).any()
    # a 0/1 panel uploaded after it carries no exception lists
    engine.upload_panel((panel == 1).astype(np.uint8))
    assert engine.exception_count() == 0


def test_stored_index_roundtrip(engine):
    # si_pbwt_save / si_pbwt_load: a ctx that loads the stored index selects and imputes as the one that built it
    from swiftimpute_b200.engine import Engine
    panel, pos, codes, _ = workload(900, 600, 30, synth.typed_every(900, 4), 100, 80)
    load(engine, panel, pos, store=False)
    blob = engine.save_index()
    assert len(blob) == 32 + 900 * 128 * 4
    pairs = {L: engine.select_states(L) for L in (8, 16)}
    want = engine.impute(codes)
    with Engine(0) as other:
        other.upload_panel(panel)
        other.set_map(pos)
        other.load_index(blob)
        for L in (8, 16):
            assert np.array_equal(other.select_states(L), pairs[L])
        got = other.impute(codes)
        assert np.array_equal(got["dosage"], want["dosage"]) and np.array_equal(got["haps"], want["haps"])
        changed = panel.copy()
        changed[450, 17] ^= 1
        other.upload_panel(changed)
        with pytest.raises(N.SIError) as e:
            other.load_index(blob)
        assert e.value.status == 1 and "different panel" in e.value.args[-1]


def test_compact_host_formats(engine):
    # 2-bit codes in and haplotype bits out give the byte path's results bit for bit
    from swiftimpute_b200.engine import pack_codes, unpack_hap_bits
    panel, pos, codes, _ = workload(700, 500, 40, synth.typed_every(700, 5), 100, 70)
    load(engine, panel, pos, store=False)
    p = N.default_params()
    full = engine.impute(codes, p)
    got = engine.impute_compact(pack_codes(codes), p, dosage=True)
    assert np.array_equal(unpack_hap_bits(got["hap_bits"], 700), full["haps"])
    assert np.array_equal(got["dosage"], full["dosage"])
    only = engine.impute_compact(pack_codes(codes), p)
    assert np.array_equal(only["hap_bits"], got["hap_bits"])
    # byte haplotypes without a dosage buffer (the posterior variant without the dosage sums)
    assert np.array_equal(engine.impute(codes, p, dosage=False)["haps"], full["haps"])
    # a panel with alleles other than 0/1 needs the byte output
    engine.upload_panel(with_other_alleles(panel, 71))
    engine.set_map(pos)
    engine.pbwt_build()
    with pytest.raises(N.SIError) as e:
        engine.impute_compact(pack_codes(codes), p)
    assert e.value.status == 4


def test_fb_unmatched_calls(engine):
    # typed calls that no selected pair can produce scale every slot alike
    panel, pos, codes, _ = workload(400, 256, 20, synth.typed_every(400, 2), 120, 11)
    codes = codes.copy()
    codes[:, ::2] = np.where(codes[:, ::2] == 3, 3, (codes[:, ::2] + 1) % 3)
    compare(engine, panel, pos, codes, 8, 10000)


@pytest.mark.parametrize("M", [1, 2, 31, 32, 33, 65])
def test_fb_short_chains(engine, M):
    panel, pos, codes, _ = workload(M, 200, 5, synth.typed_every(M, 2), 100, 12)
    compare(engine, panel, pos, codes, 8, 10000)


def test_fb_tiles_do_not_change_results(engine):
    panel, pos, codes, _ = workload(300, 400, 100, synth.typed_every(300, 5), 100, 13)
    load(engine, panel, pos, store=False)
    base = engine.impute(codes, N.default_params(), hap_prob=True)
    # typed path: C anchors per window; full chain: C markers per checkpoint segment
    tiles = {0: [(8, 32), (17, 96), (32, 64), (1, 32), (4, 128)],
             N.IMPUTE_FULL_CHAIN: [(8, 32), (17, 96), (32, 128), (1, 32)]}
    for flags, pairs in tiles.items():
        for C, T in pairs:
            alt = engine.impute(codes, N.default_params(checkpoint_interval=C, block_threads=T, flags=flags),
                                hap_prob=True)
            assert np.array_equal(alt["haps"], base["haps"])
            assert np.abs(alt["dosage"] - base["dosage"]).max() <= 2e-5
    ms = engine.last_kernel_ms()
    assert len(ms) == 4 and ms[3] > 0
    # a typed tile whose window records exceed shared memory is refused, not truncated
    with pytest.raises(N.SIError) as e:
        engine.impute(codes, N.default_params(num_states=32, checkpoint_interval=32, block_threads=128))
    assert e.value.status == 4  # SI_ERR_UNSUPPORTED


def test_fb_philox_sampling_and_batch_invariance(engine):
    panel, pos, codes, _ = workload(600, 500, 48, synth.typed_every(600, 5), 100, 14)
    got, _ = compare(engine, panel, pos, codes, 8, 10000, sampling=N.SAMPLE_PHILOX, seed=77, sid=1000)
    # a sample's draw depends only on (seed, sample id, marker), never on its batch
    p = N.default_params(sampling=N.SAMPLE_PHILOX, seed=77, sample_id_base=1000 + 5)
    alone = engine.impute(codes[5:6], p)
    assert np.array_equal(alone["haps"][0], got["haps"][5])
    assert np.array_equal(alone["dosage"][0], got["dosage"][5])


def test_fb_gl_input_equals_codes(engine):
    panel, pos, codes, _ = workload(200, 300, 10, synth.typed_every(200, 3), 100, 15)
    load(engine, panel, pos, store=False)
    a = engine.impute(codes, hap_prob=True)
    b = engine.impute(oracle.codes_to_gl(codes), gl=True, hap_prob=True)
    for k in a:
        assert np.array_equal(a[k], b[k])
    bad = oracle.codes_to_gl(codes)
    bad[0, 0] = [-0.5, -1.0, -2.0]
    with pytest.raises(N.SIError) as e:
        engine.impute(bad, gl=True)
    assert e.value.status == 4


def test_fb_codes_above_three_are_missing(engine):
    panel, pos, codes, _ = workload(100, 300, 4, synth.typed_every(100, 3), 100, 16)
    load(engine, panel, pos, store=False)
    a = engine.impute(codes)
    c2 = codes.copy()
    c2[c2 == 3] = 200
    b = engine.impute(c2)
    assert np.array_equal(a["haps"], b["haps"]) and np.array_equal(a["dosage"], b["dosage"])


def test_errors_are_reported_not_thrown(engine):
    panel, pos, codes, _ = workload(50, 100, 2, synth.typed_every(50, 3), 100, 17)
    load(engine, panel, pos, store=False)
    with pytest.raises(N.SIError) as e:
        engine.impute(codes, N.default_params(num_states=33))
    assert e.value.status == 4
    with pytest.raises(N.SIError) as e:
        engine.prefix_rows()
    assert e.value.status == 5
    # zero genetic distance gives a switch weight of exp(-999): refused, not mis-computed
    engine.set_map(np.ones(50, dtype=np.uint64))
    with pytest.raises(N.SIError) as e:
        engine.impute(codes)
    assert e.value.status == 4


def test_budget_is_enforced():
    from swiftimpute_b200.engine import Engine
    with Engine(0, hbm_budget_bytes=1 << 20) as eng:
        panel = np.zeros((4000, 4432), np.uint8)
        with pytest.raises(N.SIError) as e:
            eng.upload_panel(panel)
        assert e.value.status == 7


def test_ragged_missingness_per_sample(engine):
    """Each sample has its own typed set (random dropouts and extra calls), so
    the typed-marker kernel's anchor lists differ in length per sample."""
    panel, pos, codes, truth = workload(1200, 500, 45, synth.typed_every(1200, 6), 100, 18)
    rng = np.random.default_rng(19)
    codes = codes.copy()
    drop = rng.random(codes.shape) < 0.3
    codes[drop] = 3
    extra = rng.random(codes.shape) < 0.02
    codes[extra] = truth[extra]
    codes[3, :] = 3          # a sample with no calls at all
    codes[4, :] = truth[4]   # a sample typed everywhere
    codes[5, 0] = 3          # marker 0 missing
    compare(engine, panel, pos, codes, 8, 10000)
    compare(engine, panel, pos, codes, 16, 10000, sampling=N.SAMPLE_PHILOX)


@pytest.mark.parametrize("spacing,every", [(100, 5), (500_000, 5), (20, 97), (100, 1)])
def test_typed_kernel_agrees_with_full_chain(engine, spacing, every):
    panel, pos, codes, _ = workload(1500, 600, 64, synth.typed_every(1500, every), spacing, 20)
    load(engine, panel, pos, store=False)
    typed = engine.impute(codes, N.default_params(), hap_prob=True)
    full = engine.impute(codes, N.default_params(flags=N.IMPUTE_FULL_CHAIN), hap_prob=True)
    assert np.abs(typed["dosage"] - full["dosage"]).max() <= 2e-5
    assert np.abs(typed["hap_prob"] - full["hap_prob"]).max() <= 2e-5
    assert np.mean(typed["haps"] != full["haps"]) <= 1e-4


def test_long_untyped_gaps_beyond_tables(engine):
    """Gaps longer than the 4,096-entry closed-form tables use the on-the-fly
    formulas."""
    panel, pos, codes, _ = workload(9000, 200, 6, np.array([0, 5, 4700, 8999]), 30, 21)
    compare(engine, panel, pos, codes, 8, 10000)
    panel, pos, codes, _ = workload(9000, 200, 6, np.array([3, 4500]), 500_000, 22)
    compare(engine, panel, pos, codes, 4, 10000)


@pytest.mark.parametrize("sampling", [N.SAMPLE_ARGMAX, N.SAMPLE_PHILOX])
def test_host_buffer_call_in_chunks_equals_one_launch(engine, sampling):
    # 50,000 markers: the host-buffer call splits 2,700 targets into chunks of 1,342 (64 MB of codes)
    import torch
    panel, pos, codes, _ = workload(50_000, 400, 2700, synth.typed_every(50_000, 9), 100, 14)
    load(engine, panel, pos, store=False)
    p = N.default_params(sampling=sampling, seed=21, sample_id_base=5000)
    got = engine.impute(codes, p, hap_prob=True)
    B, M = codes.shape
    dev = torch.device("cuda", 0)
    d_geno = torch.from_numpy(codes).to(dev)
    d_dos = torch.empty((B, M), dtype=torch.float32, device=dev)
    d_hp = torch.empty((B, M, 2), dtype=torch.float32, device=dev)
    d_haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)
    engine.impute_device(d_geno.data_ptr(), B, p, d_dos.data_ptr(), d_hp.data_ptr(), d_haps.data_ptr())
    torch.cuda.synchronize(dev)
    assert np.array_equal(got["dosage"], d_dos.cpu().numpy())
    assert np.array_equal(got["hap_prob"], d_hp.cpu().numpy())
    assert np.array_equal(got["haps"], d_haps.cpu().numpy())
