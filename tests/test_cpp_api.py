"""The reference-shaped C++ API (include/swiftimpute/imputer.hpp), driven by a
compiled C++ caller (tests/cpp/api_tool.cpp)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from swiftimpute_b200 import synth
from swiftimpute_b200._native import LIB_PATH
from vcfutil import write_panel_vcf, write_target_vcf

ROOT = Path(__file__).resolve().parent.parent


def _has_device():
    import ctypes
    n = ctypes.c_int(0)
    try:
        return ctypes.CDLL("libcudart.so").cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


@pytest.fixture(scope="module")
def api_tool(tmp_path_factory):
    exe = tmp_path_factory.mktemp("bin") / "api_tool"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/api_tool.cpp"),
                    "-L", str(LIB_PATH.parent), "-lswiftimpute_b200", f"-Wl,-rpath,{LIB_PATH.parent}", "-o", str(exe)],
                   check=True)
    return exe


@pytest.fixture(scope="module")
def vcfs(tmp_path_factory):
    d = tmp_path_factory.mktemp("vcf")
    panel, pos, _ = synth.make_panel(180, 300, 10, seed=31, spacing=150)
    typed = synth.typed_every(180, 4)
    codes, _, _ = synth.make_targets(panel, 17, typed, seed=32)
    write_panel_vcf(d / "ref.vcf", panel, pos)
    write_target_vcf(d / "tgt.vcf", codes, pos)
    return d, panel, pos, codes


def test_vcf_parse_binary_roundtrip_and_writer(api_tool, vcfs):
    d, panel, pos, codes = vcfs
    r = subprocess.run([str(api_tool), "parse", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "p")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "roundtrip=1 target_roundtrip=1 refused=1" in r.stdout
    # 2 bits per target cell: a header plus ceil(M/4) bytes per sample, against 12 B per cell in memory
    B, M = codes.shape
    assert (d / "p.sitarget").stat().st_size - B * ((M + 3) // 4) < 64 * M + 64 * B
    got_panel = np.fromfile(d / "p.panel", np.uint8).reshape(panel.shape)
    assert np.array_equal(got_panel, panel)
    gl = np.fromfile(d / "p.gl", np.float32).reshape(codes.shape + (3,))
    assert np.array_equal(gl, oracle.codes_to_gl(codes))  # hard calls -> {0,-999,-999}, missing -> {0,0,0}
    lines = (d / "p.out.vcf").read_text().splitlines()
    assert lines[:3] == ["##fileformat=VCFv4.2", "##source=SwiftImpute", "##contig=<ID=chr1>"]
    assert lines[8].startswith("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\tTARGET1")
    row = lines[9].split("\t")
    assert row[:9] == ["chr1", str(int(pos[0])), "rs1", "A", "G", ".", "PASS", "IMP", "GT"]
    assert row[9] == f"{panel[0, 0]}|{panel[0, 1]}"
    assert len(lines) == 9 + panel.shape[0]


@pytest.fixture(scope="module")
def vcfs_other(tmp_path_factory):
    """A panel VCF with '.' calls (ALLELE_MISSING, 255) and allele-2 calls at multi-allelic sites."""
    d = tmp_path_factory.mktemp("vcf_other")
    panel, pos, _ = synth.make_panel(160, 300, 10, seed=33, spacing=150)
    codes, _, _ = synth.make_targets(panel, 9, synth.typed_every(160, 4), seed=34)
    rng = np.random.default_rng(35)
    u = rng.random(panel.shape)
    panel = panel.copy()
    panel[u < 0.01] = 255
    panel[(u >= 0.01) & (u < 0.015)] = 2
    write_panel_vcf(d / "ref.vcf", panel, pos)
    write_target_vcf(d / "tgt.vcf", codes, pos)
    return d, panel, pos, codes


def test_vcf_panel_with_missing_and_multiallelic_calls(api_tool, vcfs_other):
    """ReferencePanel::load_vcf keeps '.' as 255 and allele indices as they are
    (imputer.cpp:85-112); the binary panel format carries them."""
    d, panel, pos, codes = vcfs_other
    r = subprocess.run([str(api_tool), "parse", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "p")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "roundtrip=1" in r.stdout
    assert np.array_equal(np.fromfile(d / "p.panel", np.uint8).reshape(panel.shape), panel)
    assert (d / "p.sipanel").read_bytes()[:8] == b"SIPANEL2"


@pytest.mark.gpu
def test_imputer_with_missing_and_multiallelic_panel(api_tool, vcfs_other):
    d, panel, pos, codes = vcfs_other
    r = subprocess.run([str(api_tool), "impute", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "o.vcf"),
                        str(d / "o"), "1", "8", "10000", "1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    B, M = codes.shape
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)
    want = oracle.fb_batch(codes, pairs, panel, pos, 8, 10000.0)
    assert np.abs(np.fromfile(d / "o.dosage", np.float32).reshape(B, M) - want["dosage"]).max() <= 1e-4
    assert np.array_equal(np.fromfile(d / "o.haps", np.uint8).reshape(B, 2, M), want["haps_argmax"])


def test_binary_loaders_refuse_damaged_files(api_tool, vcfs):
    d, panel, pos, codes = vcfs
    r = subprocess.run([str(api_tool), "parse", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "b")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    for kind, name, shape in (("panel", "b.sipanel", f"M={panel.shape[0]} N={panel.shape[1]}"),
                              ("target", "b.sitarget", f"M={codes.shape[1]} B={codes.shape[0]}")):
        whole = (d / name).read_bytes()
        ok = subprocess.run([str(api_tool), "loadbin", kind, str(d / name)], capture_output=True, text=True)
        assert ok.returncode == 0 and shape in ok.stdout
        for cut, words in ((len(whole) - 1, "truncated"), (len(whole) // 3, "truncated"), (6, "not a")):
            (d / "damaged").write_bytes(whole[:cut])
            r = subprocess.run([str(api_tool), "loadbin", kind, str(d / "damaged")], capture_output=True, text=True)
            assert r.returncode == 11 and words in r.stdout, (kind, cut, r.stdout)
        # a damaged count in the header (haplotypes of a panel, markers of a target file): refused
        # before anything of that size is allocated
        bad = bytearray(whole)
        at = 12 if kind == "panel" else 8
        bad[at:at + 4] = b"\xff\xff\xff\x7f"
        (d / "damaged").write_bytes(bytes(bad))
        r = subprocess.run([str(api_tool), "loadbin", kind, str(d / "damaged")], capture_output=True, text=True)
        assert r.returncode == 11 and ("truncated" in r.stdout or "corrupt" in r.stdout), (kind, r.stdout)


def test_imputer_without_device_raises_cuda_error(api_tool, vcfs):
    if _has_device():
        pytest.skip("a device is visible")
    d, *_ = vcfs
    r = subprocess.run([str(api_tool), "impute", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "o.vcf"),
                        str(d / "o"), "1", "8", "10000"], capture_output=True, text=True)
    assert r.returncode == 10 and "CUDAError" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("deterministic,posteriors", [(1, 0), (0, 1)])
def test_imputer_end_to_end(api_tool, vcfs, deterministic, posteriors):
    d, panel, pos, codes = vcfs
    r = subprocess.run([str(api_tool), "impute", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "o.vcf"),
                        str(d / "o"), str(deterministic), "8", "10000", str(posteriors)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    B, M = codes.shape
    assert f"progress_calls=3 last={B}/{B}" in r.stdout  # 17 samples in passes of 7
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)
    want = oracle.fb_batch(codes, pairs, panel, pos, 8, 10000.0, sampled=not deterministic)
    ds = np.fromfile(d / "o.dosage", np.float32).reshape(B, M)
    assert np.abs(ds - want["dosage"]).max() <= 1e-4
    haps = np.fromfile(d / "o.haps", np.uint8).reshape(B, 2, M)
    if deterministic:
        assert np.array_equal(haps, want["haps_argmax"])
    else:
        assert np.mean(haps != want["haps_sampled"]) <= 1e-3
    hard = np.fromfile(d / "o.hard", np.float32).reshape(B, M)
    assert np.array_equal(hard, haps[:, 0] + haps[:, 1])  # get_dosage keeps the reference meaning
    gp = np.fromfile(d / "o.gp", np.float32).reshape(B, M, 3)
    p = want["hap_prob"]
    assert np.abs(gp[..., 2] - p[..., 0] * p[..., 1]).max() <= 2e-4
    lines = (d / "o.vcf").read_text().splitlines()
    fmt = lines[9].split("\t")[8]
    assert fmt == ("GT:DS:GP" if posteriors else "GT")
    assert len(lines) == 9 + M


@pytest.mark.gpu
def test_imputer_stored_index(api_tool, vcfs):
    """Imputer::save_index / load_index (pbwt_index.hpp:257-258): a second
    Imputer that loads the stored index gives the same haplotypes."""
    d, *_ = vcfs
    r = subprocess.run([str(api_tool), "index", str(d / "ref.vcf"), str(d / "tgt.vcf"), str(d / "p.siindex")],
                       capture_output=True, text=True)
    assert r.returncode == 0 and "index same=1 has_index=1" in r.stdout, r.stdout + r.stderr


def test_multi_gpu_imputer_refusals_without_device(api_tool, vcfs):
    d, *_ = vcfs
    args = [str(api_tool), "multi", str(d / "ref.vcf"), str(d / "tgt.vcf")]
    r = subprocess.run(args + ["", str(d / "m"), "1", "8", "10000"], capture_output=True, text=True)
    assert r.returncode == 11 and "at least one device" in r.stdout  # checked before any device call
    r = subprocess.run(args + ["0,-1", str(d / "m"), "1", "8", "10000"], capture_output=True, text=True)
    if _has_device():
        assert r.returncode == 11 and "negative" in r.stdout
    else:
        assert r.returncode == 10 and "CUDAError" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("devices,deterministic", [("0", 1), ("0,0,0", 1), ("0,0", 0)])
def test_multi_gpu_imputer_replicas_match_one_imputer(api_tool, vcfs, devices, deterministic):
    """MultiGPUImputer (src/api/imputer.hpp:298-328) as sample-sharded replicas:
    repeated device ids give several replicas on the one device here; 17
    targets split 6/6/5 (or 9/8) and the gathered result is bit-identical to one
    Imputer, argmax and Philox sampling alike."""
    d, panel, pos, codes = vcfs
    r = subprocess.run([str(api_tool), "multi", str(d / "ref.vcf"), str(d / "tgt.vcf"), devices, str(d / "m"),
                        str(deterministic), "8", "10000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"replicas={len(devices.split(','))} identical=1" in r.stdout
    B, M = codes.shape
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)
    want = oracle.fb_batch(codes, pairs, panel, pos, 8, 10000.0, sampled=not deterministic)
    ds = np.fromfile(d / "m.dosage", np.float32).reshape(B, M)
    assert np.abs(ds - want["dosage"]).max() <= 1e-4
    if deterministic:
        haps = np.fromfile(d / "m.haps", np.uint8).reshape(B, 2, M)
        assert np.array_equal(haps, want["haps_argmax"])


REF_MAIN = oracle.REFERENCE_TREE / "src" / "main.cpp"


@pytest.mark.skipif(not REF_MAIN.exists(), reason="reference source tree not present")
def test_reference_cli_compiles_unchanged(tmp_path):
    """The reference's own CLI (src/main.cpp), fed to the compiler as-is, builds
    against include/ (api/imputer.hpp, core/types.hpp forwarders) and links
    this library: the C++ API is a drop-in."""
    exe = tmp_path / "swiftimpute_cli"
    with open(REF_MAIN) as src:
        r = subprocess.run(["g++", "-std=c++17", "-x", "c++", "-I", str(ROOT / "include"), "-",
                            "-L", str(LIB_PATH.parent), "-lswiftimpute_b200", f"-Wl,-rpath,{LIB_PATH.parent}",
                            "-o", str(exe)], stdin=src, cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe), "--help"], capture_output=True, text=True)
    assert "Usage" in out.stdout
