"""CPU oracle (TEST INFRASTRUCTURE): ctypes wrappers over oracle/si_oracle.c.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg and
reference arm may import this package. It is the checker, never the thing
measured or shipped; the product library does not link it.

``ref_pbwt`` / ``ref_gpu`` expose the reference's own code compiled from its
unmodified sources into oracle/_ref/ (see oracle/Makefile) when present.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libsi_oracle.so"
REF_PBWT_SO = HERE / "_ref" / "libref_pbwt.so"
REF_GPU_SO = HERE / "_ref" / "libref_gpu.so"

# Where the reference's source tree lies when it is present (the oracle/_ref
# builds, the golden-vector generator and the drop-in compile test read it);
# SI_REFERENCE_TREE overrides. Absent on machines that only run the prebuilt files.
REFERENCE_TREE = Path(os.environ.get("SI_REFERENCE_TREE", "/root/reference"))

SEL_AUTO, SEL_WARP, SEL_INSERTION, SEL_FIRST_PAIRS = 0, 1, 2, 3
TRANS_MATRIX0, TRANS_PER_GAP = 0, 1


class FbArgs(ctypes.Structure):
    _fields_ = [("M", c_uint32), ("N", c_uint32), ("L", c_uint32), ("trans_mode", c_int),
                ("tie_eps", c_double), ("seed", c_uint64), ("sample_id", c_uint64)]


def build(target: str = "oracle") -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), target, f"REF={REFERENCE_TREE}"], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build("oracle")
        L = ctypes.CDLL(str(ORACLE_SO))
        L.sio_row_hash.restype = c_uint64
        L.sio_row_hash.argtypes = [c_void_p, c_uint32]
        L.sio_philox_u32.restype = c_uint32
        L.sio_philox_u32.argtypes = [c_uint32] * 6
        L.sio_uniform.restype = c_double
        L.sio_uniform.argtypes = [c_uint64, c_uint64, c_uint32]
        L.sio_select_kind.restype = c_int
        L.sio_select_kind.argtypes = [c_uint32, c_uint32]
        L.sio_transition_log10.argtypes = [c_double, c_double, c_double, c_double, POINTER(c_float), POINTER(c_float)]
        L.sio_pbwt_build.argtypes = [c_void_p, c_uint32, c_uint32, c_void_p]
        L.sio_pbwt_build_packed.argtypes = [c_void_p, c_uint32, c_uint32, c_uint32, c_void_p, c_void_p]
        L.sio_select_row.argtypes = [c_void_p, c_uint32, c_uint32, c_int, c_void_p]
        L.sio_select_target.argtypes = [c_void_p, c_void_p, c_void_p, c_uint32, c_uint32, c_uint32, c_void_p]
        L.sio_fb_sample.argtypes = [POINTER(FbArgs)] + [c_void_p] * 11
        L.sio_fb_batch.argtypes = [POINTER(FbArgs), c_uint32] + [c_void_p] * 10 + [c_int]
        L.sio_codes_to_gl.argtypes = [c_void_p, c_uint64, c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def pbwt_build(panel: np.ndarray) -> np.ndarray:
    panel = np.ascontiguousarray(panel, dtype=np.uint8)
    M, N = panel.shape
    out = np.empty((M, N), dtype=np.uint32)
    lib().sio_pbwt_build(_p(panel), M, N, _p(out))
    return out


def pbwt_build_packed(words: np.ndarray, N: int, keep_prefix: bool = True):
    words = np.ascontiguousarray(words, dtype=np.uint32)
    M, W = words.shape
    prefix = np.empty((M, N), dtype=np.uint32) if keep_prefix else None
    hashes = np.empty(M, dtype=np.uint64)
    lib().sio_pbwt_build_packed(_p(words), M, N, W, _p(prefix), _p(hashes))
    return prefix, hashes


def row_hash(row: np.ndarray) -> int:
    row = np.ascontiguousarray(row, dtype=np.uint32)
    return int(lib().sio_row_hash(_p(row), row.size))


def select_kind(N: int, L: int) -> int:
    return int(lib().sio_select_kind(N, L))


def select_pairs(prefix: np.ndarray, L: int, kind: int = SEL_AUTO) -> np.ndarray:
    """[M][L][2] haplotype pairs for every marker of a prefix array."""
    M, N = prefix.shape
    slots = np.empty((M, L), dtype=np.uint32)
    row = np.empty(L, dtype=np.uint32)
    pre = np.ascontiguousarray(prefix, dtype=np.uint32)
    for m in range(M):
        lib().sio_select_row(_p(pre[m]), N, L, kind, _p(row))
        slots[m] = row
    return np.stack([slots, (slots + 1) % N], axis=-1).astype(np.uint32)


def select_pairs_target(prefix: np.ndarray, panel: np.ndarray, codes: np.ndarray, L: int) -> np.ndarray:
    """[M][L][2] target-aware slot pairs of one target (codes [M]) from the full prefix array."""
    pre = np.ascontiguousarray(prefix, dtype=np.uint32)
    pan = np.ascontiguousarray(panel, dtype=np.uint8)
    cod = np.ascontiguousarray(codes, dtype=np.uint8)
    M, N = pan.shape
    out = np.empty((M, L, 2), dtype=np.uint32)
    lib().sio_select_target(_p(pre), _p(pan), _p(cod), M, N, L, _p(out))
    return out


def transition_log10(gd0: float, gd1: float, ne: float, rho_rate: float) -> tuple[float, float]:
    d, o = c_float(), c_float()
    lib().sio_transition_log10(gd0, gd1, ne, rho_rate, ctypes.byref(d), ctypes.byref(o))
    return d.value, o.value


def transitions(pos: np.ndarray, ne: float, rho_rate: float = 4.0, per_gap: bool = False):
    """(t_diag, t_off) float32 arrays: one entry (matrix 0) or M-1 entries (per gap).
    Genetic positions are pos / 1e8 Morgans (src/api/imputer.cpp:596-604)."""
    gd = pos.astype(np.float64) / 1e8
    n = (len(pos) - 1) if per_gap else 1
    td = np.empty(max(n, 1), np.float32)
    to = np.empty(max(n, 1), np.float32)
    if len(pos) < 2:
        td[0], to[0] = 0.0, -999.0
        return td, to
    for g in range(n):
        td[g], to[g] = transition_log10(gd[g], gd[g + 1], ne, rho_rate)
    return td, to


def codes_to_gl(codes: np.ndarray) -> np.ndarray:
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    gl = np.empty(codes.shape + (3,), dtype=np.float32)
    lib().sio_codes_to_gl(_p(codes), codes.size, _p(gl))
    return gl


def philox_u32(c0, c1, c2, c3, k0, k1) -> int:
    return int(lib().sio_philox_u32(c0, c1, c2, c3, k0, k1))


def uniform(seed: int, sample_id: int, marker: int) -> float:
    return float(lib().sio_uniform(seed, sample_id, marker))


def fb_batch(codes_or_gl: np.ndarray, pairs: np.ndarray, panel: np.ndarray, pos: np.ndarray, L: int, ne: float,
             rho_rate: float = 4.0, per_gap: bool = False, tie_eps: float = 1e-4, seed: int = 12345,
             sample_id_base: int = 0, threads: int | None = None, sampled: bool = False):
    """FP64 log-space forward-backward over B samples sharing one slot table.

    Returns dict with dosage [B][M], hap_prob [B][M][2], haps_argmax [B][2][M]
    and, if sampled, haps_sampled [B][2][M].
    """
    gl = codes_or_gl if codes_or_gl.dtype == np.float32 and codes_or_gl.ndim == 3 else codes_to_gl(codes_or_gl)
    gl = np.ascontiguousarray(gl, dtype=np.float32)
    B, M, _ = gl.shape
    panel = np.ascontiguousarray(panel, dtype=np.uint8)
    N = panel.shape[1]
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    td, to = transitions(pos, ne, rho_rate, per_gap)
    a = FbArgs(M, N, L, TRANS_PER_GAP if per_gap else TRANS_MATRIX0, tie_eps, seed, sample_id_base)
    dosage = np.empty((B, M), np.float32)
    p0 = np.empty((B, M), np.float32)
    p1 = np.empty((B, M), np.float32)
    ham = np.empty((B, 2, M), np.uint8)
    has = np.empty((B, 2, M), np.uint8) if sampled else None
    lib().sio_fb_batch(ctypes.byref(a), B, _p(gl), _p(pairs), _p(panel), _p(td), _p(to), _p(dosage), _p(p0),
                       _p(p1), _p(ham), _p(has), threads or os.cpu_count() or 1)
    out = {"dosage": dosage, "hap_prob": np.stack([p0, p1], axis=-1), "haps_argmax": ham}
    if sampled:
        out["haps_sampled"] = has
    return out


def fb_logpost(gl_row: np.ndarray, pairs: np.ndarray, panel: np.ndarray, pos: np.ndarray, L: int, ne: float,
               rho_rate: float = 4.0, per_gap: bool = False) -> np.ndarray:
    """Unnormalised log posterior [M][L] (alpha + beta, natural log) of one sample."""
    gl = np.ascontiguousarray(gl_row, dtype=np.float32)
    M = gl.shape[0]
    panel = np.ascontiguousarray(panel, dtype=np.uint8)
    td, to = transitions(pos, ne, rho_rate, per_gap)
    a = FbArgs(M, panel.shape[1], L, TRANS_PER_GAP if per_gap else TRANS_MATRIX0, 0.0, 0, 0)
    lp = np.empty((M, L), np.float64)
    lib().sio_fb_sample(ctypes.byref(a), _p(gl), _p(np.ascontiguousarray(pairs, dtype=np.uint32)), _p(panel),
                        _p(td), _p(to), None, None, None, None, None, _p(lp))
    return lp


# --- the reference compiled from its own sources ------------------------------

def ref_pbwt_available() -> bool:
    return REF_PBWT_SO.exists()


def ref_pbwt_build(panel: np.ndarray):
    """(prefix, divergence) from the reference's PBWTBuilder::build."""
    L = ctypes.CDLL(str(REF_PBWT_SO))
    L.ref_pbwt_build.restype = c_int
    L.ref_pbwt_build.argtypes = [c_void_p, c_uint32, c_uint32, c_void_p, c_void_p]
    panel = np.ascontiguousarray(panel, dtype=np.uint8)
    M, N = panel.shape
    pre = np.empty((M, N), np.uint32)
    div = np.empty((M, N), np.uint32)
    if L.ref_pbwt_build(_p(panel), M, N, _p(pre), _p(div)) != 0:
        raise RuntimeError("reference PBWTBuilder::build failed")
    return pre, div


def ref_gpu_available() -> bool:
    return REF_GPU_SO.exists()


def ref_gpu_impute(panel: np.ndarray, pos: np.ndarray, gl: np.ndarray, L: int, ne: int, rho_rate: float = 4.0,
                   iters: int = 1, want_logpost: bool = True):
    """Run the reference's own GPU path (compiled from source) on a B200.

    Returns (slots [M][L], logpost [B][M][L] or None, haps [B][2][M], stage_ms[4]).
    """
    Lb = ctypes.CDLL(str(REF_GPU_SO))
    Lb.ref_gpu_impute.restype = c_int
    Lb.ref_gpu_impute.argtypes = [c_void_p, c_uint32, c_uint32, c_void_p, c_void_p, c_uint32, c_uint32, c_uint32,
                                  c_float, c_int, c_void_p, c_void_p, c_void_p, c_void_p]
    panel = np.ascontiguousarray(panel, dtype=np.uint8)
    M, N = panel.shape
    gl = np.ascontiguousarray(gl, dtype=np.float32)
    B = gl.shape[0]
    slots = np.empty((M, L), np.uint32)
    lp = np.empty((B, M, L), np.float32) if want_logpost else None
    haps = np.empty((B, 2, M), np.uint8)
    ms = np.zeros(4, np.float32)
    rc = Lb.ref_gpu_impute(_p(panel), M, N, _p(np.ascontiguousarray(pos, dtype=np.uint64)), _p(gl), B, L, ne,
                           rho_rate, iters, _p(slots), _p(lp), _p(haps), _p(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU path returned {rc}")
    return slots, lp, haps, ms


def ref_gpu_fb_timing(panel: np.ndarray, pos: np.ndarray, gl: np.ndarray, L: int, ne: int, slots: np.ndarray,
                      rho_rate: float = 4.0, iters: int = 1) -> np.ndarray:
    """Stage times (ms: emission, forward+backward, sampling) of the reference's
    plain log-space kernels on a B200 over the given slot table [M][L]."""
    Lb = ctypes.CDLL(str(REF_GPU_SO))
    Lb.ref_gpu_fb_timing.restype = c_int
    Lb.ref_gpu_fb_timing.argtypes = [c_void_p, c_uint32, c_uint32, c_void_p, c_void_p, c_uint32, c_uint32, c_uint32,
                                     c_float, c_void_p, c_int, c_void_p]
    panel = np.ascontiguousarray(panel, dtype=np.uint8)
    M, N = panel.shape
    gl = np.ascontiguousarray(gl, dtype=np.float32)
    ms = np.zeros(3, np.float32)
    rc = Lb.ref_gpu_fb_timing(_p(panel), M, N, _p(np.ascontiguousarray(pos, dtype=np.uint64)), _p(gl), gl.shape[0],
                              L, ne, rho_rate, _p(np.ascontiguousarray(slots, dtype=np.uint32)), iters, _p(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU timing returned {rc}")
    return ms
