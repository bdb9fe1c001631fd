"""Write small synthetic VCFs for the C++ API tests."""
from __future__ import annotations

import numpy as np


def _allele(v) -> str:
    return "." if int(v) == 255 else str(int(v))


def write_panel_vcf(path, panel: np.ndarray, pos: np.ndarray, chrom: str = "chr1"):
    """panel [M][N] alleles (N even) as phased diploid samples REF1..REF{N/2};
    255 is written as '.', and a row with allele 2 gets a second ALT allele."""
    M, N = panel.shape
    with open(path, "w") as f:
        f.write("##fileformat=VCFv4.2\n")
        f.write(f"##contig=<ID={chrom},length={int(pos[-1]) + 1}>\n")
        f.write('##FORMAT=<ID=GT,Number=1,Type=String,Description="Genotype">\n')
        f.write("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t"
                + "\t".join(f"REF{i + 1}" for i in range(N // 2)) + "\n")
        for m in range(M):
            gts = "\t".join(f"{_allele(panel[m, 2 * s])}|{_allele(panel[m, 2 * s + 1])}" for s in range(N // 2))
            alt = "G,T" if (panel[m] == 2).any() else "G"
            f.write(f"{chrom}\t{int(pos[m])}\trs{m + 1}\tA\t{alt}\t100\tPASS\t.\tGT\t{gts}\n")


def write_target_vcf(path, codes: np.ndarray, pos: np.ndarray, chrom: str = "chr1"):
    """codes [B][M] (0/1/2, 3 = missing) as unphased genotypes TARGET1..TARGET{B}."""
    B, M = codes.shape
    txt = {0: "0/0", 1: "0/1", 2: "1/1", 3: "./."}
    with open(path, "w") as f:
        f.write("##fileformat=VCFv4.2\n")
        f.write(f"##contig=<ID={chrom},length={int(pos[-1]) + 1}>\n")
        f.write('##FORMAT=<ID=GT,Number=1,Type=String,Description="Genotype">\n')
        f.write("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t"
                + "\t".join(f"TARGET{i + 1}" for i in range(B)) + "\n")
        for m in range(M):
            gts = "\t".join(txt[int(codes[b, m])] for b in range(B))
            f.write(f"{chrom}\t{int(pos[m])}\trs{m + 1}\tA\tG\t100\tPASS\t.\tGT\t{gts}\n")
