"""The large-panel workload at full size: 100,000 haplotypes x 100,000
markers (bit-packed, 1.25 GB), 500 founders, switch rate 0.001; 50,000 targets
typed at every 20th marker (5 %), L = 16, uniform 0.5 cM map.

The panel and targets are generated on the device with torch (a host-side
byte panel would take 10 GB and minutes to draw); the generator follows the
same recipe as swiftimpute_b200.synth (founder mosaic with allele flips;
targets a mosaic of 8 panel haplotypes with switch rate 0.005), without the
heterozygosity resampling. Checks:
  * the PBWT sweep equals the oracle's streaming sweep row by row (64-bit
    hash of every prefix row, all 100,000 rows);
  * every output of all 50,000 targets is finite and in range;
  * dosage and argmax haplotypes of a seeded subset of 512 targets equal the
    FP64 oracle (1e-4; argmax up to threshold flips), on the 0.5 cM map and
    on a 1 kb map. The oracle reads the
    device's slot table through a compact panel of the 32 selected haplotype
    columns per marker, which gives it the same emissions as the full panel.
"""
import numpy as np
import pytest

import oracle
from swiftimpute_b200 import _native as N

pytestmark = pytest.mark.gpu

M = NH = 100_000
B = 50_000
L = 16
NE = 10_000
EVERY = 20


def _panel(dev):
    from swiftimpute_b200 import synth_device
    return synth_device.make_panel(M, NH, 500, (0.5, 0.5), 0.001, 0.005, seed=3, device=dev)


def _pack(panel):
    from swiftimpute_b200 import synth_device
    return synth_device.pack_panel(panel)


def _targets(panel):
    from swiftimpute_b200 import synth_device
    return synth_device.make_targets(panel, B, EVERY, seed=3)


@pytest.fixture(scope="module")
def large(engine):
    import torch
    dev = torch.device("cuda", 0)
    panel = _panel(dev)
    words = _pack(panel)
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(500_000)).astype(np.uint64)
    engine.upload_packed(words, NH)
    engine.set_map(pos)
    engine.pbwt_build(row_hashes=True)
    codes = _targets(panel)
    yield panel, words, pos, codes
    del panel, codes
    torch.cuda.empty_cache()


def test_pbwt_rows_equal_oracle_streaming_sweep(engine, large):
    _, words, _, _ = large
    _, want = oracle.pbwt_build_packed(words, NH, keep_prefix=False)
    assert np.array_equal(engine.row_hashes(), want)


def _impute_and_check_subset(engine, large, pos, name):
    import torch
    panel, _, _, codes = large
    dev = codes.device
    params = N.default_params(num_states=L, ne=NE)
    dos = torch.empty((B, M), dtype=torch.float32, device=dev)
    haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)
    engine.impute_device(codes.data_ptr(), B, params, dos.data_ptr(), None, haps.data_ptr())
    torch.cuda.synchronize(dev)
    assert bool(torch.isfinite(dos).all()) and float(dos.min()) >= -1e-6 and float(dos.max()) <= 2 + 1e-5
    assert int(haps.max()) <= 1
    # seeded subset against the oracle, through a compact panel of the selected columns
    sub = np.sort(np.random.default_rng(3).choice(B, 512, replace=False))
    pairs = engine.select_states(L)                                        # [M][L][2]
    cols = torch.from_numpy(pairs.reshape(M, 2 * L).astype(np.int64)).to(dev)
    compact = torch.gather(panel, 1, cols).cpu().numpy()                   # [M][2L] alleles of the slot pairs
    cpairs = np.broadcast_to(np.arange(2 * L, dtype=np.uint32).reshape(1, L, 2), (M, L, 2)).copy()
    idx = torch.from_numpy(sub).to(dev)
    c_sub = codes.index_select(0, idx).cpu().numpy()
    got_d = dos.index_select(0, idx).cpu().numpy()
    got_h = haps.index_select(0, idx).cpu().numpy()
    del dos, haps
    torch.cuda.empty_cache()
    want = oracle.fb_batch(c_sub, cpairs, compact, pos, L, float(NE))
    from conftest import r2_masked, report
    r2 = r2_masked(got_d, want["dosage"], c_sub)
    report(name, targets=512,
           max_abs_dosage_diff=np.abs(got_d - want["dosage"]).max(), dosage_r2_vs_oracle=r2,
           argmax_cells_differing=int((got_h != want["haps_argmax"]).sum()), cells=int(512 * M))
    assert r2 >= 1 - 1e-6
    assert np.abs(got_d - want["dosage"]).max() <= 1e-4
    diff = (got_h != want["haps_argmax"]).any(axis=1)
    if diff.any():
        rows = np.nonzero(diff.any(axis=1))[0]
        lo = oracle.fb_batch(c_sub[rows], cpairs, compact, pos, L, float(NE), tie_eps=1e-4 - 1e-5)
        hi = oracle.fb_batch(c_sub[rows], cpairs, compact, pos, L, float(NE), tie_eps=1e-4 + 1e-5)
        flip = ((lo["haps_argmax"] != want["haps_argmax"][rows]) | (hi["haps_argmax"] != want["haps_argmax"][rows])).any(axis=1)
        assert not (diff[rows] & ~flip).any()


def test_all_targets_and_oracle_subset(engine, large):
    _impute_and_check_subset(engine, large, large[2], "large panel 100,000 x 100,000, 0.5 cM map, 512 targets")


def test_dense_map_oracle_subset(engine, large):
    # markers 1 kb apart: the transition keeps memory (rho < 1)
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(1000)).astype(np.uint64)
    engine.set_map(pos)
    _impute_and_check_subset(engine, large, pos, "large panel 100,000 x 100,000, 1 kb map, 512 targets")
