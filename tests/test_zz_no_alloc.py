"""The allocation-free entry point, si_impute_device_noalloc.

It serves callers that cannot call cudaMalloc when they impute: programs whose
device memory belongs to another allocator (a framework's pool), and
latency-bound programs sharing the device with other streams, where an
allocation may synchronise the device. Its checkpoint scratch is a fixed array
inside the library. These tests call it through the C ABI twice in a row, with
different inputs, and check each result against the allocating entry point
si_impute_device within the parity tolerance of the other GPU tests (dosage
and P(hap=1) 1e-4; haplotypes may differ only at argmax near-ties, <= 1e-4 of
cells). Each test creates its own context, so the file passes alone in a fresh
process as well as after the other tests.
"""
from ctypes import byref, c_uint64, c_void_p

import numpy as np
import pytest

from swiftimpute_b200 import _native as N
from swiftimpute_b200 import synth
from swiftimpute_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-4
ERR_INVALID_ARG, ERR_UNSUPPORTED, ERR_STATE = 1, 4, 5


def _ckpt_bytes(B, M, L, C):
    """Checkpoint scratch of one call: max(ceil(M / C) - 1, 1) * Lmax * B * 4."""
    lmax = 4 if L <= 4 else 8 if L <= 8 else 16 if L <= 16 else 32
    nseg = (M + C - 1) // C
    return max(nseg - 1, 1) * lmax * B * 4


def _run_two_calls(torch, num_states, use_stream):
    dev = torch.device("cuda", 0)
    M, Nh, B = 1500, 600, 96
    panel, pos, _ = synth.make_panel(M, Nh, 16, seed=41, spacing=100)
    typed = synth.typed_every(M, 5)
    codes_a, _, _ = synth.make_targets(panel, B, typed, seed=42)
    codes_b, _, _ = synth.make_targets(panel, B, typed, seed=43)
    C = 16 if num_states > 16 else 32
    need = _ckpt_bytes(B, M, num_states, C)
    with Engine(0) as eng:
        eng.upload_panel(panel)
        eng.set_map(pos)
        eng.pbwt_build()
        p = N.default_params(num_states=num_states, ne=10000)
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
        stream = torch.cuda.Stream(dev) if use_stream else None
        handle = c_void_p(stream.cuda_stream) if stream is not None else None
        # Two calls in a row. The first call on the ctx is its set-up: it looks
        # up the scratch array's address, and with lazy module loading that is
        # when the driver commits the array itself. The ctx's own accounting
        # must not move, and the device's free memory must not drop by anything
        # like the checkpoints the call needs (an allocation of them would show).
        used0 = c_uint64()
        eng._check(lib.si_ctx_memory(eng.h, byref(used0), None))
        free_after_first = None
        for name in ("a", "b"):
            g, ref, new = outs[name]
            st = lib.si_impute_device_noalloc(eng.h, byref(p), c_void_p(g.data_ptr()), B,
                                              c_void_p(new[0].data_ptr()), c_void_p(new[1].data_ptr()),
                                              c_void_p(new[2].data_ptr()), handle)
            assert st == N.SI_OK, lib.si_last_error(eng.h).decode()
            if stream is not None:
                stream.synchronize()
            torch.cuda.synchronize(dev)
            if free_after_first is None:
                free_after_first = torch.cuda.mem_get_info(0)[0]
        assert free_after_first - torch.cuda.mem_get_info(0)[0] < need // 2
        used1 = c_uint64()
        eng._check(lib.si_ctx_memory(eng.h, byref(used1), None))
        assert used1.value == used0.value
        for name in ("a", "b"):
            g, ref, new = outs[name]
            d_ref, d_new = ref[0].cpu().numpy(), new[0].cpu().numpy()
            assert np.abs(d_new - d_ref).max() <= TOL
            assert np.abs(new[1].cpu().numpy() - ref[1].cpu().numpy()).max() <= TOL
            assert np.mean(new[2].cpu().numpy() != ref[2].cpu().numpy()) <= 1e-4
        return eng, p, outs


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    _run_two_calls(torch, 8, use_stream=False)


def test_noalloc_on_caller_stream_with_32_slots():
    torch = pytest.importorskip("torch")
    _run_two_calls(torch, 32, use_stream=True)


def test_noalloc_refusals():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    M, Nh, B = 600, 300, 16
    panel, pos, _ = synth.make_panel(M, Nh, 12, seed=44, spacing=100)
    codes, _, _ = synth.make_targets(panel, B, synth.typed_every(M, 5), seed=45)
    with Engine(0) as eng:
        eng.upload_panel(panel)
        eng.set_map(pos)
        eng.pbwt_build()
        p = N.default_params(num_states=8, ne=10000)
        lib = eng.lib
        g = torch.from_numpy(codes).to(dev)
        dos = torch.empty((B, M), dtype=torch.float32, device=dev)
        # before any allocating call the tables are missing
        st = lib.si_impute_device_noalloc(eng.h, byref(p), c_void_p(g.data_ptr()), B,
                                          c_void_p(dos.data_ptr()), None, None, None)
        assert st == ERR_STATE
        eng.impute_device(g.data_ptr(), B, p, dos.data_ptr(), 0, 0)
        torch.cuda.synchronize(dev)
        # sizes beyond the fixed scratch are refused with a clear error
        st = lib.si_impute_device_noalloc(eng.h, byref(p), c_void_p(g.data_ptr()), 200_000,
                                          c_void_p(dos.data_ptr()), None, None, None)
        assert st == ERR_UNSUPPORTED and b"scratch" in lib.si_last_error(eng.h)
        # unknown flag bits are refused, as by si_impute_device
        q = N.default_params(num_states=8, ne=10000)
        q.flags = 0x100
        st = lib.si_impute_device_noalloc(eng.h, byref(q), c_void_p(g.data_ptr()), B,
                                          c_void_p(dos.data_ptr()), None, None, None)
        assert st == ERR_INVALID_ARG
