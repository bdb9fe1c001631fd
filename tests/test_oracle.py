"""The CPU oracle against the reference's own code and against a second,
pure-Python restatement of the recurrences (CPU only)."""
import math

import numpy as np
import pytest

import oracle
from swiftimpute_b200 import synth


@pytest.mark.skipif(not oracle.ref_pbwt_available(), reason="reference PBWT not built (oracle/_ref)")
@pytest.mark.parametrize("M,N,seed,p1", [(10, 8, 0, 0.5), (257, 333, 1, 0.3), (600, 4432, 2, 0.1), (50, 1, 3, 0.5)])
def test_pbwt_matches_reference_builder(M, N, seed, p1):
    rng = np.random.default_rng(seed)
    panel = (rng.random((M, N)) < p1).astype(np.uint8)
    pre_ref, div_ref = oracle.ref_pbwt_build(panel)
    assert np.array_equal(oracle.pbwt_build(panel), pre_ref)
    # the reference's divergence array is m in every entry of row m
    assert np.array_equal(div_ref, np.broadcast_to(np.arange(M, dtype=np.uint32)[:, None], (M, N)))


@pytest.mark.skipif(not oracle.ref_pbwt_available(), reason="reference PBWT not built (oracle/_ref)")
def test_pbwt_missing_alleles_sort_as_one():
    rng = np.random.default_rng(9)
    panel = (rng.random((40, 100)) < 0.4).astype(np.uint8)
    panel[3, ::3] = 255  # ALLELE_MISSING goes to the non-zero side (pbwt_index.cpp:183)
    assert np.array_equal(oracle.pbwt_build(panel), oracle.ref_pbwt_build(panel)[0])


def test_packed_sweep_equals_u8_sweep():
    rng = np.random.default_rng(5)
    panel = (rng.random((120, 777)) < 0.35).astype(np.uint8)
    pre_u8 = oracle.pbwt_build(panel)
    pre_pk, hashes = oracle.pbwt_build_packed(synth.pack_panel(panel), 777)
    assert np.array_equal(pre_u8, pre_pk)
    assert hashes[7] == oracle.row_hash(pre_u8[7])
    assert len(set(hashes.tolist())) == len(hashes)


def test_selection_patterns():
    N = 300
    row = np.arange(N, dtype=np.uint32)[::-1].copy()
    pairs = oracle.select_pairs(row[None, :], 8, oracle.SEL_WARP)[0]
    assert pairs[:, 0].tolist() == [row[0], row[32], row[64], row[96], 4, 5, 6, 7]
    assert pairs[:, 1].tolist() == [(h + 1) % N for h in pairs[:, 0].tolist()]
    ins = oracle.select_pairs(row[None, :], 8, oracle.SEL_INSERTION)[0]
    assert ins[:, 0].tolist() == row[:8].tolist()
    # kernel choice as launch_select_states
    assert oracle.select_kind(4432, 8) == oracle.SEL_WARP
    assert oracle.select_kind(100000, 16) == oracle.SEL_INSERTION
    assert oracle.select_kind(4432, 48) == oracle.SEL_INSERTION
    # fewer haplotypes than the pattern: lane 0 holds ceil(N/32) entries; fill i % N
    small = np.arange(40, dtype=np.uint32)[None, :]
    s = oracle.select_pairs(small, 6, oracle.SEL_WARP)[0][:, 0].tolist()
    assert s == [0, 32, 2, 3, 4, 5]
    s = oracle.select_pairs(np.arange(5, dtype=np.uint32)[None, :], 8, oracle.SEL_INSERTION)[0][:, 0].tolist()
    assert s == [0, 1, 2, 3, 4, 5 % 5, 6 % 5, 7 % 5]


def test_transition_uniform_under_half_cM_map():
    # 0.5 cM spacing: rho = 1 - exp(-16 Ne d) clamps to 1, so stay == switch
    d, o = oracle.transition_log10(0.0, 0.005, 10000.0, 4.0)
    assert d == o == np.float32(math.log10(1.0 / 20000.0))
    d, o = oracle.transition_log10(0.0, 1e-6, 10000.0, 4.0)
    rho = 1 - math.exp(-16 * 10000 * 1e-6)
    assert d == np.float32(math.log10(1 - rho + rho / 20000)) and o == np.float32(math.log10(rho / 20000))
    d, o = oracle.transition_log10(0.0, 0.0, 10000.0, 4.0)
    assert (d, o) == (0.0, -999.0)


def test_philox_known_answers():
    # Random123 philox4x32-10 known-answer vectors (first output word)
    assert oracle.philox_u32(0, 0, 0, 0, 0, 0) == 0x6627E8D5
    assert oracle.philox_u32(*([0xFFFFFFFF] * 6)) == 0x408F276D
    assert oracle.philox_u32(0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344, 0xA4093822, 0x299F31D0) == 0xD16CFE09
    u = [oracle.uniform(12345, 7, m) for m in range(1000)]
    assert min(u) >= 0.0 and max(u) < 1.0 and abs(np.mean(u) - 0.5) < 0.05


def _lse2(a, b):
    m = max(a, b)
    return math.log(math.exp(a - m) + math.exp(b - m)) + m


def python_logpost(gl, pairs, panel, td, to, L):
    """Second restatement, plain Python loops (forward_backward.cu:41-317)."""
    M = gl.shape[0]

    def E(m, k):
        s = int(panel[m, pairs[m, k, 0]]) + int(panel[m, pairs[m, k, 1]])
        return float(gl[m, 0 if s == 0 else (1 if s == 1 else 2)])

    T = lambda i, j: float(td if i == j else to)
    alpha = [[E(0, k) for k in range(L)]]
    mx = max(alpha[0]); alpha[0] = [x - mx for x in alpha[0]]
    for m in range(1, M):
        row = []
        for j in range(L):
            s = -999.0
            for i in range(L):
                s = _lse2(s, alpha[-1][i] + T(i, j))
            row.append(s + E(m, j))
        mx = max(row); alpha.append([x - mx for x in row])
    beta = [[0.0] * L for _ in range(M)]
    for m in range(M - 2, -1, -1):
        for i in range(L):
            s = -999.0
            for j in range(L):
                s = _lse2(s, (T(i, j) + E(m + 1, j)) + beta[m + 1][j])
            beta[m][i] = s
    return np.array([[alpha[m][k] + beta[m][k] for k in range(L)] for m in range(M)])


@pytest.mark.parametrize("spacing,L", [(100, 3), (500_000, 4), (2, 5)])
def test_oracle_fb_matches_python_restatement(spacing, L):
    panel, pos, _ = synth.make_panel(25, 64, 6, seed=11, spacing=spacing)
    typed = synth.typed_every(25, 3)
    codes, _, _ = synth.make_targets(panel, 2, typed, seed=12)
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)
    gl = oracle.codes_to_gl(codes)
    td, to = oracle.transitions(pos, 10000.0)
    for b in range(2):
        lp = oracle.fb_logpost(gl[b], pairs, panel, pos, L, 10000.0)
        ref = python_logpost(gl[b], pairs, panel, td[0], to[0], L)
        assert np.allclose(lp, ref, rtol=0, atol=1e-9)


def test_oracle_floor_regime():
    """Long untyped runs push beta to the e^-999 floor; posteriors stay finite
    and the dosage keeps to [0, 2]."""
    panel, pos, _ = synth.make_panel(900, 200, 8, seed=2, spacing=500_000)
    typed = np.array([0, 10, 450, 899])
    codes, _, _ = synth.make_targets(panel, 3, typed, seed=3)
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)
    lp = oracle.fb_logpost(oracle.codes_to_gl(codes)[0], pairs, panel, pos, 8, 10000.0)
    assert np.isfinite(lp).all() and lp.min() < -900  # beta reached the floor
    out = oracle.fb_batch(codes, pairs, panel, pos, 8, 10000.0)
    assert np.all((out["dosage"] >= 0) & (out["dosage"] <= 2))
    assert np.allclose(out["dosage"], out["hap_prob"].sum(-1), atol=1e-6)


def _target_pairs_bruteforce(panel, prefix, codes, L):
    """Target-aware slots by explicit key comparison: the target's position at
    marker m is the number of haplotypes whose reversed prefix (alleles m, m-1,
    ..., 0, non-zero as 1) sorts strictly before the target's, whose own
    alleles are its homozygous calls and elsewhere the allele of the haplotype
    at its previous position (the last one when it sits past the end)."""
    M, N = panel.shape
    bits = (panel != 0).astype(np.int64)
    tgt = []
    p = 0
    out = np.empty((M, L, 2), dtype=np.uint32)
    for m in range(M):
        prev = prefix[m - 1] if m else np.arange(N)
        hq = prev[min(p, N - 1)]
        tgt.append(0 if codes[m] == 0 else 1 if codes[m] == 2 else int(bits[m, hq]))
        tkey = tgt[::-1]
        p = 0
        for h in range(N):
            if list(bits[m::-1, h]) < tkey:
                p += 1
        s0 = min(max(p - L // 2, 0), N - L) if L <= N else 0
        for r in range(L):
            h = int(prefix[m][s0 + r]) if L <= N else int(prefix[m][r % N])
            out[m, r] = (h, (h + 1) % N)
    return out


@pytest.mark.parametrize("M,N,L,seed", [(30, 20, 4, 0), (25, 33, 8, 1), (20, 6, 8, 2), (40, 16, 16, 3)])
def test_target_selection_matches_key_sort(M, N, L, seed):
    rng = np.random.default_rng(seed)
    panel = (rng.random((M, N)) < 0.4).astype(np.uint8)
    prefix = oracle.pbwt_build(panel)
    for _ in range(4):
        codes = rng.integers(0, 4, size=M).astype(np.uint8)
        assert np.array_equal(oracle.select_pairs_target(prefix, panel, codes, L),
                              _target_pairs_bruteforce(panel, prefix, codes, L))
