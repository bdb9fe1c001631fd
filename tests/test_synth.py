"""Seeded generator: shapes, determinism and the stated distributions (CPU)."""
import numpy as np

from swiftimpute_b200 import synth


def test_deterministic_and_shapes():
    a = synth.plain_small(seed=0, B=12, M=300, N=500)
    b = synth.plain_small(seed=0, B=12, M=300, N=500)
    assert np.array_equal(a.panel, b.panel) and np.array_equal(a.codes, b.codes)
    assert a.panel.shape == (300, 500) and a.codes.shape == (12, 300)
    assert set(np.unique(a.panel)) <= {0, 1}
    assert np.all(a.codes[:, a.typed] == a.truth[:, a.typed])
    masked = np.setdiff1d(np.arange(300), a.typed)
    assert np.all(a.codes[:, masked] == synth.MISSING)
    assert a.imputed_cells == 12 * (300 - 60)
    assert int(a.pos[1] - a.pos[0]) == 500_000


def test_heterozygosity_window():
    panel, _, _ = synth.make_panel(400, 800, 40, seed=4)
    _, truth, haps = synth.make_targets(panel, 50, synth.typed_every(400, 5), seed=5)
    het = (haps[:, 0] != haps[:, 1]).mean(axis=1)
    assert np.all((het >= 0.12) & (het <= 0.40))


def test_pack_panel_bit_order():
    rng = np.random.default_rng(0)
    p = (rng.random((3, 70)) < 0.5).astype(np.uint8)
    w = synth.pack_panel(p)
    assert w.shape == (3, 3)
    for m in range(3):
        for h in range(70):
            assert ((int(w[m, h // 32]) >> (h % 32)) & 1) == p[m, h]


def test_typed_evenly():
    t = synth.typed_evenly(50_000, 3000)
    assert t.size == 3000 and t[0] == 0 and t[-1] < 50_000
