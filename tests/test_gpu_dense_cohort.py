"""The dense-cohort workload at full size on a map with memory: a 4,432 x
50,000 panel (100 founders), 10,000 targets typed at 3,000 evenly spaced
markers, L = 8, Ne = 20,000, markers 1 kb apart (rho = 1 - exp(-16 Ne d)
stays below 1, so the transition is not the memoryless one the 0.5 cM map
gives, transition.cu:91-96).

All 10,000 targets are imputed on the device; 768 from the start and the
last 256 (ending in the batch's partial 32-sample group, whose chain warp
also runs lanes past the batch's end) are checked against the FP64 oracle
(dosage and P(hap=1) within 1e-4, argmax haplotypes bit-exact except at
threshold flips), and the last 1,000 imputed alone match the full batch bit
for bit. Panel and targets come from the device
generator (swiftimpute_b200.synth_device) with the workload's shapes.
"""
import numpy as np
import pytest

import oracle
from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth, synth_device

pytestmark = pytest.mark.gpu

M, NH, B, NTYPED, L, NE = 50_000, 4432, 10_000, 3000, 8, 20_000
CHECK = 1024
ROWS = np.r_[0:768, B - 256:B]  # the batch's start and its end (partial last group)


@pytest.mark.parametrize("spacing", [1000])
def test_dense_cohort_full_size_against_oracle(engine, spacing):
    import torch
    dev = torch.device("cuda", 0)
    panel_d = synth_device.make_panel(M, NH, 100, seed=11, device=dev)
    typed = synth.typed_evenly(M, NTYPED)
    codes_d = synth_device.make_targets(panel_d, B, typed=typed, seed=11)
    panel = panel_d.cpu().numpy()
    del panel_d
    pos = (1 + np.arange(M, dtype=np.uint64) * np.uint64(spacing)).astype(np.uint64)
    engine.upload_panel(panel)
    engine.set_map(pos)
    engine.pbwt_build()
    params = N.default_params(num_states=L, ne=NE)
    dos = torch.empty((B, M), dtype=torch.float32, device=dev)
    hp = torch.empty((B, M, 2), dtype=torch.float32, device=dev)
    haps = torch.empty((B, 2, M), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)
    engine.impute_device(codes_d.data_ptr(), B, params, dos.data_ptr(), hp.data_ptr(), haps.data_ptr())
    torch.cuda.synchronize(dev)
    assert bool(torch.isfinite(dos).all()) and float(dos.min()) >= -1e-6 and float(dos.max()) <= 2 + 1e-5
    # batch invariance: the last 1,000 targets alone
    tail = B - 1000
    dos1 = torch.empty((1000, M), dtype=torch.float32, device=dev)
    hp1 = torch.empty((1000, M, 2), dtype=torch.float32, device=dev)
    haps1 = torch.empty((1000, 2, M), dtype=torch.uint8, device=dev)
    p1 = N.default_params(num_states=L, ne=NE)
    p1.sample_id_base = tail
    engine.impute_device(codes_d[tail:].data_ptr(), 1000, p1, dos1.data_ptr(), hp1.data_ptr(), haps1.data_ptr())
    torch.cuda.synchronize(dev)
    assert torch.equal(dos1, dos[tail:]) and torch.equal(hp1, hp[tail:]) and torch.equal(haps1, haps[tail:])
    del dos1, hp1, haps1
    rows = torch.from_numpy(ROWS).to(dev)
    codes = codes_d[rows].cpu().numpy()
    got_d = dos[rows].cpu().numpy()
    got_p = hp[rows].cpu().numpy()
    got_h = haps[rows].cpu().numpy()
    pairs = engine.select_states(L)
    want = oracle.fb_batch(codes, pairs, panel, pos, L, float(NE))
    dd = np.abs(got_d - want["dosage"]).max()
    dp = np.abs(got_p - want["hap_prob"]).max()
    from conftest import r2_masked, report
    r2 = r2_masked(got_d, want["dosage"], codes)
    report(f"dense cohort full size, {spacing} bp map", targets=CHECK, max_abs_dosage_diff=dd,
           max_abs_hap_prob_diff=dp, dosage_r2_vs_oracle=r2,
           argmax_cells_differing=int((got_h != want["haps_argmax"]).sum()), cells=int(CHECK * M))
    assert dd <= 1e-4, f"max |d dosage| = {dd}"
    assert dp <= 1e-4, f"max |d P(hap=1)| = {dp}"
    assert r2 >= 1 - 1e-6
    diff = (got_h != want["haps_argmax"]).any(axis=1)
    if diff.any():
        rows = np.nonzero(diff.any(axis=1))[0]
        lo = oracle.fb_batch(codes[rows], pairs, panel, pos, L, float(NE), tie_eps=1e-4 - 1e-5)
        hi = oracle.fb_batch(codes[rows], pairs, panel, pos, L, float(NE), tie_eps=1e-4 + 1e-5)
        flip = ((lo["haps_argmax"] != want["haps_argmax"][rows]) | (hi["haps_argmax"] != want["haps_argmax"][rows])).any(axis=1)
        assert not (diff[rows] & ~flip).any(), "argmax cells differ away from the tie threshold"
