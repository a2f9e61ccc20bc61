"""The walk kernel finds a hop's Green-CDF bin from the Philox word w itself
(walk.cu, bin_of_word): guide entry w >> 24, then integer tests
w > ceil(intg[k] * 2^32) - 1, instead of the FP64 search on u = w / 2^32
(bin_of: guide entry floor(u * 256), then intg[k] <= u).  This checks, on the
CPU with the product's Green table, that both give the same bin for every
one of the 2^32 words."""
import shutil
import subprocess

import numpy as np
import pytest

import frw

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#define NS 200
int main(void) {
    double intg[NS + 1];
    if (fread(intg, sizeof(double), NS + 1, stdin) != NS + 1) return 2;
    uint8_t guide[256];
    for (int k = 0; k < 256; k++) {  /* the kernel's guide: binary search of k / 256 */
        const double u = (double)k * (1.0 / 256);
        int lo = 0, hi = NS;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (intg[mid] <= u) lo = mid; else hi = mid;
        }
        guide[k] = (uint8_t)lo;
    }
    uint32_t thr[NS + 1];
    for (int k = 0; k <= NS; k++) thr[k] = (uint32_t)((unsigned long long)ceil(intg[k] * 0x1p32) - 1ull);
    uint64_t bad = 0;
    for (uint64_t w64 = 0; w64 < (1ull << 32); w64++) {
        const uint32_t w = (uint32_t)w64;
        const double u = (double)w * 0x1p-32;
        int a = guide[(int)(u * 256.0)];
        while (a < NS - 1 && intg[a + 1] <= u) a++;
        int b = guide[w >> 24];
        while (b < NS - 1 && w > thr[b + 1]) b++;
        bad += a != b;
    }
    printf("%llu\n", (unsigned long long)bad);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_integer_bin_search_equals_fp64_search_for_every_word(tmp_path):
    _, intg = frw.green_table()
    src = tmp_path / "bins.c"
    exe = tmp_path / "bins"
    src.write_text(SRC)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(src), "-lm"], check=True)
    out = subprocess.run([str(exe)], input=np.ascontiguousarray(intg, dtype=np.float64).tobytes(),
                         capture_output=True, check=True, timeout=600)
    assert int(out.stdout.decode().strip()) == 0
