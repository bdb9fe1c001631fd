"""The allocation-free entry point, si_impute_device_noalloc.

It serves callers that cannot call cudaMalloc when they impute: code inside
CUDA stream capture (an allocation there synchronises the device and breaks
the capture) and programs whose device memory belongs to another allocator.
Its checkpoint scratch is a fixed array inside the library. This test calls
it through the C ABI twice in a row, with different inputs, and checks each
result against the allocating entry point si_impute_device within the parity
tolerance of the other GPU tests (dosage and P(hap=1) 1e-4; haplotypes may
differ only at argmax near-ties, <= 1e-4 of cells). It creates its own
context so it passes alone in a fresh process as well as after other tests.
"""
import ctypes
from ctypes import byref, c_uint64, c_void_p

import numpy as np
import pytest

from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth
from swiftimpute_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _device_free_bytes(torch):
    free, _ = torch.cuda.mem_get_info(0)
    return free


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    M, Nh, B = 1500, 600, 96
    panel, pos, _ = synth.make_panel(M, Nh, 16, seed=41, spacing=100)
    typed = synth.typed_every(M, 5)
    codes_a, _, _ = synth.make_targets(panel, B, typed, seed=42)
    codes_b, _, _ = synth.make_targets(panel, B, typed, seed=43)
    with Engine(0) as eng:
        eng.upload_panel(panel)
        eng.set_map(pos)
        eng.pbwt_build()
        p = N.default_params(num_states=8, ne=10000)
        lib = eng.lib
        outs = {}
        for name, codes in (("a", codes_a), ("b", codes_b)):
            g = torch.from_numpy(codes).to(dev)
            ref = (torch.empty((B, M), dtype=torch.float32, device=dev),
                   torch.empty((B, M, 2), dtype=torch.float32, device=dev),
                   torch.empty((B, 2, M), dtype=torch.uint8, device=dev))
            new = (torch.empty_like(ref[0]), torch.empty_like(ref[1]), torch.empty_like(ref[2]))
            eng.impute_device(g.data_ptr(), B, p, ref[0].data_ptr(), ref[1].data_ptr(), ref[2].data_ptr())
            torch.cuda.synchronize(dev)
            outs[name] = (g, ref, new)
        # two calls in a row on the allocation-free path. The first call on the
        # device is its set-up: it looks up the scratch array's address, and with
        # lazy module loading that is when the driver commits the array itself.
        # After it, calls must leave the device's free memory unchanged.
        used0 = c_uint64()
        eng._check(lib.si_ctx_memory(eng.h, byref(used0), None))
        free_after_first = None
        for name in ("a", "b"):
            g, ref, new = outs[name]
            st = lib.si_impute_device_noalloc(eng.h, byref(p), c_void_p(g.data_ptr()), B,
                                              c_void_p(new[0].data_ptr()), c_void_p(new[1].data_ptr()),
                                              c_void_p(new[2].data_ptr()), None)
            assert st == N.SI_OK, lib.si_last_error(eng.h).decode()
            torch.cuda.synchronize(dev)
            if free_after_first is None:
                free_after_first = _device_free_bytes(torch)
        assert _device_free_bytes(torch) == free_after_first
        used1 = c_uint64()
        eng._check(lib.si_ctx_memory(eng.h, byref(used1), None))
        assert used1.value == used0.value
        for name in ("a", "b"):
            g, ref, new = outs[name]
            d_ref, d_new = ref[0].cpu().numpy(), new[0].cpu().numpy()
            assert np.abs(d_new - d_ref).max() <= TOL
            assert np.abs(new[1].cpu().numpy() - ref[1].cpu().numpy()).max() <= TOL
            assert np.mean(new[2].cpu().numpy() != ref[2].cpu().numpy()) <= 1e-4
        # sizes beyond the fixed scratch are refused with a clear error
        big = 200_000
        st = lib.si_impute_device_noalloc(eng.h, byref(p), c_void_p(outs["a"][0].data_ptr()), big,
                                          c_void_p(outs["a"][2][0].data_ptr()), None, None, None)
        assert st == 4 and b"scratch" in lib.si_last_error(eng.h)
