"""The device kernel's reformulation, emulated in float64 on the CPU: linear
space, rank-1-plus-diagonal transition, per-marker rescaling, and beta's
absolute scale carried so the reference's e^-999 logsumexp seed (the floor)
is reproduced, switching units to e^-999 when the floor dominates. It must
equal the FP64 log-space oracle (a restatement of the reference's own
recurrences) to round-off, including deep in the floor regime."""
import math

import numpy as np
import pytest

import oracle
from swiftimpute_b200 import synth


def emulate(codes, pairs, panel, pos, L, ne):
    M = codes.shape[0]
    td, to = oracle.transitions(pos, ne)
    c = math.exp(float(to[0])); d = math.exp(float(td[0])); dl = d - c
    a0 = panel[np.arange(M)[:, None], pairs[:, :, 0]].astype(int)
    a1 = panel[np.arange(M)[:, None], pairs[:, :, 1]].astype(int)

    def em(m):
        g = int(codes[m])
        if g >= 3:
            return np.ones(L), 0
        e = ((a0[m] + a1[m]) == g).astype(float)
        return (np.ones(L), 1) if e.sum() == 0 else (e, 0)

    al = np.zeros((M, L))
    al[0] = em(0)[0]
    for m in range(1, M):
        e, _ = em(m)
        v = e * (c * al[m - 1].sum() + dl * al[m - 1])
        al[m] = v / v.sum()
    be, logs = np.ones(L), 0.0
    post = np.zeros((M, L))
    post[M - 1] = al[M - 1]
    for m in range(M - 2, -1, -1):
        e, sh = em(m + 1)
        w = e * be
        u = c * w.sum() + dl * w
        logs_u = logs - 999.0 * sh
        farg = -999.0 - logs_u
        if farg > 0:
            v, logs_new = 1.0 + math.exp(-farg) * u, -999.0
        else:
            v, logs_new = (math.exp(farg) if farg > -700 else 0.0) + u, logs_u
        s = v.sum()
        be, logs = v / s, logs_new + math.log(s)
        post[m] = al[m] * be
    return post / post.sum(1, keepdims=True)


@pytest.mark.parametrize("spacing,every,M", [(100, 5, 900), (500_000, 5, 400), (30, 50, 1200), (100, 2, 600)])
def test_scaled_recursion_equals_log_space_oracle(spacing, every, M):
    panel, pos, _ = synth.make_panel(M, 300, 12, seed=M + every, spacing=spacing)
    codes, _, _ = synth.make_targets(panel, 2, synth.typed_every(M, every), seed=3)
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)
    gl = oracle.codes_to_gl(codes)
    deep = False
    for b in range(2):
        lp = oracle.fb_logpost(gl[b], pairs, panel, pos, 8, 10000.0)
        P = np.exp(lp - lp.max(1, keepdims=True)); P /= P.sum(1, keepdims=True)
        Q = emulate(codes[b], pairs, panel, pos, 8, 10000.0)
        assert np.abs(P - Q).max() < 1e-9
        deep |= bool(lp.min() < -1500)
    if spacing == 100 and every == 5:
        assert deep  # the case reaches the floor regime with unmatched calls on top


def _floor_tables(spacing, L, ne=20000.0, NT=4096):
    """G[n] = log sum_{k=1..n} rho^-k of the run tables, rho = delta + L c of the map's first gap,
    in FP64 as the host builds them (three regimes of rho)."""
    pos = 1 + np.arange(3, dtype=np.uint64) * np.uint64(spacing)
    td, to = oracle.transitions(pos, ne)
    c = float(np.float32(math.exp(float(to[0]))))
    dl = float(np.float32(float(np.float32(math.exp(float(td[0])))) - c))
    rho = dl + L * c
    lr = math.log(rho)
    regime = 2 if abs(rho - 1.0) < 1e-15 else (0 if rho < 1.0 else 1)
    lgc = math.log1p(-rho) if regime == 0 else (math.log(rho - 1.0) if regime == 1 else 0.0)
    n = np.arange(1, NT, dtype=np.float64)
    if regime == 0:
        G = -n * lr + np.log(-np.expm1(n * lr)) - lgc
    elif regime == 1:
        G = np.log(-np.expm1(-n * lr)) - lgc
    else:
        G = np.log(n)
    return G


@pytest.mark.parametrize("spacing", [30, 1000, 500_000])
@pytest.mark.parametrize("L", [4, 8, 32])
def test_floor_log_as_float_pairs(spacing, L):
    """The posterior forms a cell's floor log farg' + G(j) in FP32 as (hi + hi) + (lo + lo),
    farg' and G(j) each split into a float and the float of its remainder. Wherever the floor
    can matter (sum in [-120, 80]) that is within 1 ulp of the FP64 sum rounded to FP32, for
    every table entry j and run constants drawn over that window."""
    G = _floor_tables(spacing, L)
    hi = G.astype(np.float32)
    lo = (G - hi.astype(np.float64)).astype(np.float32)
    rng = np.random.default_rng(spacing + L)
    for _ in range(8):
        fa = rng.uniform(-120.0, 80.0, size=G.size) - G
        fah = fa.astype(np.float32)
        fal = (fa - fah.astype(np.float64)).astype(np.float32)
        ft = (fah + hi) + (fal + lo)
        ref = (fa + G).astype(np.float32)
        err = np.abs(ft.astype(np.float64) - ref.astype(np.float64))
        assert (err <= np.spacing(np.abs(ref)).astype(np.float64)).all()


def _anchor_steps(M, spacing, every, L=8, seed=0):
    """Emission masks at the typed markers of one target and the closed-form run coefficients
    {Q_n, S_n} between consecutive typed markers (the chain's step maps)."""
    panel, pos, _ = synth.make_panel(M, 300, 12, seed=seed + M, spacing=spacing)
    typed = synth.typed_every(M, every)
    codes, _, _ = synth.make_targets(panel, 1, typed, seed=seed + 3)
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)
    td, to = oracle.transitions(pos, 20000.0)
    c = math.exp(float(to[0])); d = math.exp(float(td[0])); dl = d - c
    q = dl / (dl + L * c)
    alt = (panel[np.arange(M)[:, None], pairs[:, :, 0]].astype(int)
           + panel[np.arange(M)[:, None], pairs[:, :, 1]].astype(int))
    E = (alt[typed] == codes[0, typed][:, None]).astype(np.float64)
    E[E.sum(1) == 0] = 1.0  # no slot matches the call: every slot scaled alike
    Q = q ** np.diff(typed).astype(np.float64)
    return E, Q, (1.0 - Q) / L


def _forward(E, Q, S, dt, x, k0, k1, out):
    for k in range(k0 + 1, k1 + 1):
        x = (E[k] * (dt(Q[k - 1]) * x + dt(S[k - 1]) * x.sum())).astype(dt)
        x /= x.sum()
        out[k] = x
    return x


@pytest.mark.parametrize("spacing,every", [(100, 5), (1000, 17), (30, 3), (500_000, 5)])
def test_forward_segment_products_fp32(spacing, every):
    """Chunked parallel-in-time form of the forward chain over typed anchors: each segment's
    8 x 8 product of step maps D_k (Q_n I + S_n 11^T) in FP32 (rescaled by its maximum), the
    segment starts by a short sequential pass of products, then every segment re-run from its
    start. Its alpha stays as close to the FP64 sequential chain as the FP32 sequential chain
    is, at 8 and 64 segments."""
    E, Q, S = _anchor_steps(20_000, spacing, every)
    K, L = E.shape
    ref = np.empty((K, L)); ref[0] = E[0] / E[0].sum()
    _forward(E, Q, S, np.float64, ref[0], 0, K - 1, ref)
    seq = np.empty((K, L), np.float32); seq[0] = ref[0]
    _forward(E, Q, S, np.float32, seq[0].copy(), 0, K - 1, seq)
    err_seq = np.abs(seq - ref).max()
    for nseg in (8, 64):
        b = np.linspace(0, K - 1, nseg + 1).astype(int)
        x = seq[0].copy()
        out = np.empty((K, L), np.float32); out[0] = x
        starts = [x]
        for s in range(nseg):
            P = np.eye(L, dtype=np.float32)
            for k in range(b[s] + 1, b[s + 1] + 1):
                P = (E[k][:, None] * (np.float32(Q[k - 1]) * P + np.float32(S[k - 1]) * P.sum(0)[None, :]))
                P = (P / P.max()).astype(np.float32)
            x = (P @ x).astype(np.float32); x /= x.sum()
            starts.append(x)
        for s in range(nseg):
            out[b[s]] = starts[s]
            _forward(E, Q, S, np.float32, starts[s].copy(), b[s], b[s + 1], out)
        err = np.abs(out - ref).max()
        assert err <= max(2.0 * err_seq, 1e-7), (nseg, err, err_seq)


def _combine(v1, l1, v2, l2):
    """e^l1 v1 + e^l2 v2 as (v, l) with max(v) = 1, FP32 vectors and FP64 logs."""
    if l1 < l2:
        v1, l1, v2, l2 = v2, l2, v1, l1
    v = v1 if (l2 == -math.inf or l1 - l2 > 104.0) else (v1 + np.float32(math.exp(l2 - l1)) * v2).astype(np.float32)
    mx = float(v.max())
    return (v / np.float32(mx)).astype(np.float32), l1 + math.log(mx)


@pytest.mark.parametrize("spacing,every,M", [(100, 5, 900), (500_000, 5, 400), (30, 50, 1200), (100, 2, 600)])
def test_backward_segment_maps_with_floor_fp32(spacing, every, M):
    """Chunked parallel-in-time form of the backward chain with the reference's e^-999 floor.
    In absolute units a step is affine, beta_m = e^(-999 sh) T diag(E_m+1) beta_m+1 + e^-999 1,
    so a segment composes to beta_start = e^a A beta_end + e^bs b: A (L x L) and b in FP32 with
    their logs a, bs in FP64, the floor column merged like the sequential step (dropped beyond
    e^104). Applied from the chain's end one segment at a time, it lands on the FP64 sequential
    chain's state (unit-sum w and log U) at every segment start."""
    panel, pos, _ = synth.make_panel(M, 300, 12, seed=M + every, spacing=spacing)
    codes, _, _ = synth.make_targets(panel, 1, synth.typed_every(M, every), seed=3)
    L = 8
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), L)
    td, to = oracle.transitions(pos, 10000.0)
    c = math.exp(float(to[0])); dl = math.exp(float(td[0])) - c
    alt = (panel[np.arange(M)[:, None], pairs[:, :, 0]].astype(int)
           + panel[np.arange(M)[:, None], pairs[:, :, 1]].astype(int))
    E, SH = np.ones((M, L)), np.zeros(M, int)
    for m in range(M):
        if codes[0, m] < 3:
            e = (alt[m] == codes[0, m]).astype(float)
            if e.sum() == 0:
                SH[m] = 1
            else:
                E[m] = e
    # FP64 sequential chain (the kernel's reformulation, equal to the log-space oracle above)
    ref_w, ref_l = np.empty((M, L)), np.empty(M)
    be, logs = np.ones(L) / L, math.log(L)
    ref_w[M - 1], ref_l[M - 1] = be, logs
    for m in range(M - 2, -1, -1):
        u = c * (E[m + 1] * be).sum() + dl * E[m + 1] * be
        lu = logs - 999.0 * SH[m + 1]
        f = -999.0 - lu
        v, ln = (1.0 + math.exp(-f) * u, -999.0) if f > 0 else ((math.exp(f) if f > -700 else 0.0) + u, lu)
        be, logs = v / v.sum(), ln + math.log(v.sum())
        ref_w[m], ref_l[m] = be, logs
    T = (np.float32(c) * np.ones((L, L)) + np.float32(dl) * np.eye(L)).astype(np.float32)
    for nseg in (4, 16):
        bnd = np.linspace(0, M - 1, nseg + 1).astype(int)
        w, lw = ref_w[M - 1].astype(np.float32), ref_l[M - 1]
        for s in range(nseg - 1, -1, -1):
            A, a, b, bs = np.eye(L, dtype=np.float32), 0.0, np.zeros(L, np.float32), -math.inf
            for m in range(bnd[s + 1] - 1, bnd[s] - 1, -1):
                Ai = (T * E[m + 1][None, :]).astype(np.float32)
                A = (Ai @ A).astype(np.float32)
                mx = float(A.max())
                A, a = (A / np.float32(mx)).astype(np.float32), a - 999.0 * SH[m + 1] + math.log(mx)
                if bs > -math.inf:
                    v = (Ai @ b).astype(np.float32)
                    mv = float(v.max())
                    b, bs = _combine((v / np.float32(mv)).astype(np.float32), bs - 999.0 * SH[m + 1] + math.log(mv),
                                     np.ones(L, np.float32), -999.0)
                else:
                    b, bs = np.ones(L, np.float32), -999.0
            v = (A @ w).astype(np.float32)
            mv = float(v.max())
            v, lv = _combine((v / np.float32(mv)).astype(np.float32), a + lw + math.log(mv), b, bs)
            sm = float(v.sum())
            w, lw = (v / np.float32(sm)).astype(np.float32), lv + math.log(sm)
            assert np.abs(w - ref_w[bnd[s]]).max() <= 1e-6
            assert abs(lw - ref_l[bnd[s]]) <= 1e-4
