"""The walk's bin spacing v = perimeter / 200 for an integer perimeter is
computed on the device as q0 = x * RN(1/200) refined by one fused step with
the exact residual (query.cuh, div200).  This checks, on the CPU with the same
IEEE operations, that the refined quotient equals the correctly rounded
division for every integer x in [0, 2^31) -- the whole range an int-truncated
perimeter can take."""
import shutil
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
int main(void) {
    const double r = 1.0 / 200.0;
    uint64_t bad = 0;
    for (uint64_t k = 0; k < (1ull << 31); k++) {
        const double x = (double)k;
        const double q0 = x * r;
        const double q1 = fma(fma(-q0, 200.0, x), r, q0);
        if (q1 != x / 200.0) bad++;
    }
    printf("%llu\n", (unsigned long long)bad);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_div200_equals_division_for_every_int31(tmp_path):
    c = tmp_path / "div200.c"
    c.write_text(SRC)
    exe = tmp_path / "div200"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(c), "-lm"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=300).stdout
    assert out.strip() == "0"
