"""Python handle on a device context (thin layer over the C ABI).

``Engine`` owns one ``si_ctx``: the bit-packed panel, the PBWT index and the
selection caches stay resident on the device between calls, as the reference
``Imputer`` keeps its panel copies and index (src/api/imputer.hpp:235-259).
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_uint64, c_void_p

import numpy as np

from . import _native as N


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(c_void_p)


def _job_layout(regions, jobs):
    """Per-job code counts and offsets of an uneven batch. Every job's codes
    must cover its region exactly: the device reads the region's length from
    the job's offset, so a shorter array would be read past its end. Jobs of
    an unknown region get length 0 (the C ABI refuses them)."""
    lens = []
    for i, (r, c, _) in enumerate(jobs):
        n = max(0, regions[r][1] - regions[r][0]) if 0 <= r < len(regions) else 0
        if np.asarray(c).size != n:
            raise ValueError(f"job {i}: {np.asarray(c).size} codes for a region of {n} markers")
        lens.append(n)
    return lens, np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)


class Engine:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = N.load()
        h = c_void_p()
        st = self.lib.si_ctx_create(device, hbm_budget_bytes, byref(h))
        if st != N.SI_OK:
            raise N.SIError(st, "si_ctx_create failed (is a CUDA device visible?)")
        self.h = h
        self.device = device
        self.M = self.N = 0

    # -- plumbing -------------------------------------------------------------
    def _check(self, st: int) -> None:
        if st != N.SI_OK:
            raise N.SIError(st, self.lib.si_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.si_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def memory(self) -> tuple[int, int]:
        used, budget = c_uint64(), c_uint64()
        self._check(self.lib.si_ctx_memory(self.h, byref(used), byref(budget)))
        return used.value, budget.value

    # -- panel ----------------------------------------------------------------
    def upload_panel(self, panel: np.ndarray) -> None:
        panel = np.ascontiguousarray(panel, dtype=np.uint8)
        M, N_ = panel.shape
        self._check(self.lib.si_panel_upload_u8(self.h, _ptr(panel), M, N_))
        self.M, self.N = M, N_

    def save_index(self) -> bytes:
        """The built PBWT index in its stored form (si_pbwt_save)."""
        n = c_uint64()
        self._check(self.lib.si_pbwt_stored_bytes(self.h, byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._check(self.lib.si_pbwt_save(self.h, _ptr(buf), n.value))
        return buf.tobytes()

    def load_index(self, blob: bytes) -> None:
        """Load a stored index for the uploaded panel (si_pbwt_load)."""
        buf = np.frombuffer(blob, np.uint8)
        self._check(self.lib.si_pbwt_load(self.h, _ptr(buf), buf.size))

    def exception_count(self) -> int:
        """Panel entries other than 0 and 1 (missing or multi-allelic) of the uploaded panel."""
        n = c_uint64()
        self._check(self.lib.si_panel_exception_count(self.h, byref(n)))
        return n.value

    def upload_packed(self, words: np.ndarray, n_haplotypes: int) -> None:
        words = np.ascontiguousarray(words, dtype=np.uint32)
        M, W = words.shape
        self._check(self.lib.si_panel_upload_packed(self.h, _ptr(words), M, n_haplotypes, W))
        self.M, self.N = M, n_haplotypes

    def set_map(self, pos: np.ndarray, cM: np.ndarray | None = None) -> None:
        pos = np.ascontiguousarray(pos, dtype=np.uint64)
        cm = None if cM is None else np.ascontiguousarray(cM, dtype=np.float64)
        self._check(self.lib.si_panel_set_map(self.h, _ptr(pos), _ptr(cm)))

    # -- PBWT -------------------------------------------------------------------
    def pbwt_build(self, store_index: bool = False, row_hashes: bool = False) -> float:
        flags = (N.PBWT_STORE_INDEX if store_index else 0) | (N.PBWT_ROW_HASHES if row_hashes else 0)
        self._check(self.lib.si_pbwt_build(self.h, flags))
        ms = c_float()
        self._check(self.lib.si_pbwt_last_ms(self.h, byref(ms)))
        return ms.value

    def prefix_rows(self, m0: int = 0, count: int | None = None) -> np.ndarray:
        count = self.M - m0 if count is None else count
        out = np.empty((count, self.N), dtype=np.uint32)
        self._check(self.lib.si_pbwt_get_prefix_rows(self.h, m0, count, _ptr(out)))
        return out

    def row_hashes(self) -> np.ndarray:
        out = np.empty(self.M, dtype=np.uint64)
        self._check(self.lib.si_pbwt_row_hashes(self.h, _ptr(out)))
        return out

    # -- selection ----------------------------------------------------------------
    def select_states(self, L: int, kind: int = N.SEL_AUTO, m0: int = 0, m1: int | None = None) -> np.ndarray:
        m1 = self.M if m1 is None else m1
        out = np.empty((m1 - m0, L, 2), dtype=np.uint32)
        self._check(self.lib.si_select_states(self.h, L, kind, m0, m1, _ptr(out)))
        return out

    def select_states_target(self, L: int, codes: np.ndarray) -> np.ndarray:
        """Target-aware (SI_SEL_TARGET) slot pairs [B][M][L][2] of targets codes [B][M]."""
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        out = np.empty((codes.shape[0], codes.shape[1], L, 2), dtype=np.uint32)
        self._check(self.lib.si_select_states_target(self.h, L, _ptr(codes), codes.shape[0], _ptr(out)))
        return out

    # -- imputation ---------------------------------------------------------------
    def impute_compact(self, codes2: np.ndarray, params: N.ImputeParams | None = None, *, dosage: bool = False):
        """Impute from 2-bit packed codes ([B][ceil(M/4)], see pack_codes) and
        return bit-packed haplotypes ([B][2][ceil(M/32)] u32, see unpack_hap_bits)
        and, when asked, the dosage."""
        params = params or N.default_params()
        p = N.ImputeParams.from_buffer_copy(params)
        p.flags |= N.IMPUTE_CODES_2BIT | N.IMPUTE_HAPS_BITS
        codes2 = np.ascontiguousarray(codes2, dtype=np.uint8)
        if codes2.ndim != 2 or codes2.shape[1] != (self.M + 3) // 4:
            raise ValueError(f"codes must have shape [B][{(self.M + 3) // 4}]")
        B = codes2.shape[0]
        bits = np.empty((B, 2, (self.M + 31) // 32), np.uint32)
        d = np.empty((B, self.M), np.float32) if dosage else None
        self._check(self.lib.si_impute(self.h, byref(p), _ptr(codes2), B, _ptr(d), None, _ptr(bits)))
        out = {"hap_bits": bits}
        if dosage:
            out["dosage"] = d
        return out

    def impute(self, geno: np.ndarray, params: N.ImputeParams | None = None, *, dosage: bool = True,
               hap_prob: bool = False, haps: bool = True, gl: bool = False):
        """Impute rows of ``geno`` ([B][M] codes, or [B][M][3] log10 GL when gl=True).

        Returns a dict of numpy arrays: dosage [B][M], hap_prob [B][M][2],
        haps [B][2][M] (only the requested ones).
        """
        params = params or N.default_params()
        geno = np.ascontiguousarray(geno, dtype=np.float32 if gl else np.uint8)
        want = (self.M, 3) if gl else (self.M,)
        if geno.ndim != 1 + len(want) or geno.shape[1:] != want:
            raise ValueError(f"geno must have shape [B]{list(want)}, got {list(geno.shape)}")
        B = geno.shape[0]
        out = {}
        d = np.empty((B, self.M), np.float32) if dosage else None
        hp = np.empty((B, self.M, 2), np.float32) if hap_prob else None
        hh = np.empty((B, 2, self.M), np.uint8) if haps else None
        fn = self.lib.si_impute_gl if gl else self.lib.si_impute
        self._check(fn(self.h, byref(params), _ptr(geno), B, _ptr(d), _ptr(hp), _ptr(hh)))
        if dosage:
            out["dosage"] = d
        if hap_prob:
            out["hap_prob"] = hp
        if haps:
            out["haps"] = hh
        return out

    def impute_device(self, d_geno: int, B: int, params: N.ImputeParams, d_dosage: int | None,
                      d_hap_prob: int | None, d_haps: int | None, stream: int | None = None) -> None:
        """Queue an imputation on device buffers (raw device addresses)."""
        self._check(self.lib.si_impute_device(self.h, byref(params), c_void_p(d_geno), B,
                                              c_void_p(d_dosage) if d_dosage else None,
                                              c_void_p(d_hap_prob) if d_hap_prob else None,
                                              c_void_p(d_haps) if d_haps else None,
                                              c_void_p(stream) if stream else None))

    def impute_jobs(self, regions, jobs, params: N.ImputeParams | None = None, *, hap_prob: bool = False,
                    dosage: bool = True, stream: int | None = None):
        """Uneven batch. ``regions``: list of (m_begin, m_end, L, index_origin);
        ``jobs``: list of (region, codes[len] u8, sample_id). Outputs are packed per
        job; returns a list of dicts (dosage [len] unless ``dosage`` is false,
        haps [2][len], hap_prob [len][2]). Device buffers are allocated with torch
        (plumbing only)."""
        import torch
        params = params or N.default_params()
        R = (N.Region * len(regions))(*[N.Region(a, b, L, o) for a, b, L, o in regions])
        lens, offs = _job_layout(regions, jobs)
        J = (N.Job * len(jobs))(*[N.Job(r, 0, int(offs[i]), int(offs[i]), int(sid))
                                  for i, (r, _, sid) in enumerate(jobs)])
        total = max(1, int(offs[-1]))
        geno = np.concatenate([np.asarray(c, dtype=np.uint8).ravel() for _, c, _ in jobs] + [np.zeros(1, np.uint8)])
        dev = torch.device("cuda", self.device)
        d_geno = torch.from_numpy(geno).to(dev)
        d_dos = torch.empty(total, dtype=torch.float32, device=dev) if dosage else None
        d_haps = torch.empty(2 * total, dtype=torch.uint8, device=dev)
        d_hp = torch.empty(2 * total, dtype=torch.float32, device=dev) if hap_prob else None
        torch.cuda.synchronize(dev)
        self._check(self.lib.si_impute_jobs_device(self.h, byref(params), R, len(regions), J, len(jobs),
                                                   c_void_p(d_geno.data_ptr()),
                                                   c_void_p(d_dos.data_ptr()) if dosage else None,
                                                   c_void_p(d_hp.data_ptr()) if hap_prob else None,
                                                   c_void_p(d_haps.data_ptr()),
                                                   c_void_p(stream) if stream else None))
        torch.cuda.synchronize(dev)
        dos, haps = (d_dos.cpu().numpy() if dosage else None), d_haps.cpu().numpy()
        hp = d_hp.cpu().numpy() if hap_prob else None
        out = []
        for i in range(len(jobs)):
            a, n = int(offs[i]), lens[i]
            o = {"haps": haps[2 * a:2 * a + 2 * n].reshape(2, n)}
            if dosage:
                o["dosage"] = dos[a:a + n]
            if hap_prob:
                o["hap_prob"] = hp[2 * a:2 * a + 2 * n].reshape(n, 2)
            out.append(o)
        return out

    def plan(self, regions, jobs, params: N.ImputeParams | None = None, *, max_anchors: int = 0,
             autotune: bool = False, hap_prob: bool = False) -> "Plan":
        """A fixed uneven batch (si_plan_*): same arguments as ``impute_jobs``."""
        return Plan(self, regions, jobs, params or N.default_params(), max_anchors, autotune, hap_prob)

    def last_kernel_ms(self) -> tuple[float, float, float, float]:
        """(selection, typed-marker lists, anchor chain, posterior or full-chain kernel) in ms."""
        ms = (c_float * 4)()
        self._check(self.lib.si_last_kernel_ms(self.h, ms))
        return tuple(ms)

    def last_timings(self) -> tuple[float, float, float]:
        ms = (c_float * 3)()
        self._check(self.lib.si_last_timings(self.h, ms))
        return tuple(ms)


class Server:
    """Request queue with continuous batching over an Engine's resident panel
    and index (the si_serve_* C ABI). While it runs, the Engine must not be
    used for anything else; ``stop()`` hands it back.

    ``submit`` copies nothing: it keeps the request's code array and its output
    arrays alive until ``wait``/``poll`` reports the request finished.
    """

    def __init__(self, engine: Engine, params: N.ImputeParams | None = None, *, max_batch_cells: int = 0,
                 max_wait_us: int = 0, max_queue: int = 0, max_batch_requests: int = 0):
        self.engine = engine
        self.lib = engine.lib
        self.params = params or N.default_params()
        cfg = N.ServeConfig(max_batch_cells, max_wait_us, max_queue, max_batch_requests, 0)
        h = c_void_p()
        engine._check(self.lib.si_serve_start(engine.h, byref(self.params), byref(cfg), byref(h)))
        self.h = h
        self._held = {}

    def submit(self, m_begin: int, m_end: int, codes: np.ndarray, *, num_states: int = 8,
               index_origin: int = N.INDEX_REGION, sample_id_base: int = 0, hap_prob: bool = False,
               out: dict | None = None) -> int:
        """Queue a request; ``out`` may hold caller-owned output arrays
        (dosage [n][len] f32, haps [n][2][len] u8, hap_prob [n][len][2] f32)."""
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        n, length = codes.shape
        if length != m_end - m_begin:
            raise ValueError("codes must have m_end - m_begin columns")
        if out is None:
            out = {"dosage": np.empty((n, length), np.float32), "haps": np.empty((n, 2, length), np.uint8)}
            if hap_prob:
                out["hap_prob"] = np.empty((n, length, 2), np.float32)
        shapes = {"dosage": ((n, length), np.float32), "haps": ((n, 2, length), np.uint8),
                  "hap_prob": ((n, length, 2), np.float32)}
        for key, arr in out.items():
            if arr.shape != shapes[key][0] or arr.dtype != shapes[key][1] or not arr.flags.c_contiguous:
                raise ValueError(f"out[{key!r}] must be a C-contiguous {shapes[key][1].__name__} {shapes[key][0]}")
        req = N.Request(m_begin, m_end, num_states, index_origin, n, 0, sample_id_base, _ptr(codes),
                        _ptr(out["dosage"]), _ptr(out["haps"]), _ptr(out.get("hap_prob")))
        t = c_uint64()
        st = self.lib.si_serve_submit(self.h, byref(req), byref(t))
        if st != N.SI_OK:
            raise N.SIError(st, "request refused")
        self._held[t.value] = (codes, out)
        return t.value

    def _collect(self, ticket: int, status: int):
        codes, out = self._held.pop(ticket)
        if status != N.SI_OK:
            raise N.SIError(status, f"request {ticket} finished with an error")
        return out

    def poll(self, ticket: int):
        """None while the request runs, else its outputs (raises SIError on failure)."""
        fin, st = ctypes.c_int(), ctypes.c_int()
        s = self.lib.si_serve_poll(self.h, ticket, byref(fin), byref(st))
        if s != N.SI_OK:
            raise N.SIError(s, "unknown ticket")
        return self._collect(ticket, st.value) if fin.value else None

    def wait(self, ticket: int, timeout_ms: int = 0):
        st = ctypes.c_int()
        s = self.lib.si_serve_wait(self.h, ticket, timeout_ms, byref(st))
        if s != N.SI_OK:
            raise N.SIError(s, "wait failed" if s != 6 else "timed out")
        return self._collect(ticket, st.value)

    def cancel(self, ticket: int) -> bool:
        """True if the request was still queued and is now cancelled."""
        return self.lib.si_serve_cancel(self.h, ticket) == N.SI_OK

    def stats(self) -> dict:
        s = N.ServeStatistics()
        self.engine._check(self.lib.si_serve_stats(self.h, byref(s)))
        return {name: getattr(s, name) for name, _ in N.ServeStatistics._fields_}

    def stop(self) -> None:
        if getattr(self, "h", None):
            self.lib.si_serve_stop(self.h)
            self.h = None
            self._held.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()


class Plan:
    """A fixed uneven batch whose launch needs no host work (CUDA-graph
    capturable). Owns the device buffers of its codes and outputs (torch,
    plumbing only); ``set_codes`` rewrites the codes in place between launches."""

    def __init__(self, engine: Engine, regions, jobs, params, max_anchors, autotune, hap_prob):
        import torch
        self.engine, self.lib = engine, engine.lib
        self.regions = list(regions)
        self.lens, self.offs = _job_layout(regions, jobs)
        total = max(1, int(self.offs[-1]))
        dev = torch.device("cuda", engine.device)
        self.d_geno = torch.zeros(total, dtype=torch.uint8, device=dev)
        self.d_dos = torch.empty(total, dtype=torch.float32, device=dev)
        self.d_haps = torch.empty(2 * total, dtype=torch.uint8, device=dev)
        self.d_hp = torch.empty(2 * total, dtype=torch.float32, device=dev) if hap_prob else None
        self.set_codes([c for _, c, _ in jobs])
        R = (N.Region * len(regions))(*[N.Region(a, b, L, o) for a, b, L, o in regions])
        J = (N.Job * len(jobs))(*[N.Job(r, 0, int(self.offs[i]), int(self.offs[i]), int(sid))
                                  for i, (r, _, sid) in enumerate(jobs)])
        h = c_void_p()
        torch.cuda.synchronize(dev)
        engine._check(self.lib.si_plan_create(
            engine.h, byref(params), R, len(regions), J, len(jobs), max_anchors, c_void_p(self.d_geno.data_ptr()),
            c_void_p(self.d_dos.data_ptr()), c_void_p(self.d_hp.data_ptr()) if hap_prob else None,
            c_void_p(self.d_haps.data_ptr()), N.PLAN_AUTOTUNE if autotune else 0, byref(h)))
        self.h = h

    def set_codes(self, codes) -> None:
        import torch
        codes = [np.asarray(c, dtype=np.uint8).ravel() for c in codes]
        if [c.size for c in codes] != list(self.lens):
            raise ValueError("set_codes needs one code array per job, each as long as its region")
        flat = np.concatenate(codes) if codes else np.zeros(0, np.uint8)
        self.d_geno[: flat.size].copy_(torch.from_numpy(flat))
        torch.cuda.synchronize(self.d_geno.device)

    def launch(self, graph: bool = False, stream: int | None = None) -> None:
        fn = self.lib.si_plan_graph_launch if graph else self.lib.si_plan_launch
        self.engine._check(fn(self.h, c_void_p(stream) if stream else None))

    def check(self) -> None:
        self.engine._check(self.lib.si_plan_check(self.h))

    def info(self) -> dict:
        c, t, ms = ctypes.c_uint32(), ctypes.c_uint32(), c_float()
        self.engine._check(self.lib.si_plan_info(self.h, byref(c), byref(t), byref(ms)))
        return {"window": c.value, "threads": t.value, "tuned_ms": ms.value}

    def outputs(self):
        """Per job: dosage [len], haps [2][len] (and hap_prob [len][2])."""
        self.check()
        dos, haps = self.d_dos.cpu().numpy(), self.d_haps.cpu().numpy()
        hp = self.d_hp.cpu().numpy() if self.d_hp is not None else None
        out = []
        for i, n in enumerate(self.lens):
            a = int(self.offs[i])
            o = {"dosage": dos[a:a + n], "haps": haps[2 * a:2 * a + 2 * n].reshape(2, n)}
            if hp is not None:
                o["hap_prob"] = hp[2 * a:2 * a + 2 * n].reshape(n, 2)
            out.append(o)
        return out

    def destroy(self) -> None:
        if getattr(self, "h", None):
            self.lib.si_plan_destroy(self.h)
            self.h = None


def pack_codes(codes: np.ndarray) -> np.ndarray:
    """[B][M] genotype codes (0..3) -> [B][ceil(M/4)] bytes, cell m at bits 2 (m % 4) of byte m / 4."""
    codes = np.asarray(codes, dtype=np.uint8)
    B, M = codes.shape
    pad = np.zeros((B, 4 * ((M + 3) // 4)), np.uint8)
    pad[:, :M] = codes & 3
    q = pad.reshape(B, -1, 4)
    return (q[..., 0] | (q[..., 1] << 2) | (q[..., 2] << 4) | (q[..., 3] << 6)).astype(np.uint8)


def unpack_hap_bits(bits: np.ndarray, M: int) -> np.ndarray:
    """[B][2][ceil(M/32)] u32 words -> [B][2][M] alleles (0/1)."""
    bits = np.asarray(bits, dtype=np.uint32)
    b = np.unpackbits(bits.view(np.uint8).reshape(bits.shape[:-1] + (-1,)), axis=-1, bitorder="little")
    return b[..., :M].astype(np.uint8)
