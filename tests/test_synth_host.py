"""Host side of the seeded frame generator: the PCG32 jump-ahead the device renderer uses to reach
each pixel's draws equals stepping the generator, and the host renderer built on the shared plan
still writes the pinned frames (the golden fixtures check their hashes)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r"""
#include <stdio.h>
#include "synth_common.h"
int main(void) {
    pcg32_t r;
    pcg32_seed(&r, 987654321ULL, 0x9e3779b97f4a7c15ULL);
    pcg32_t a = r;
    for (unsigned long long d = 0; d < 200000; ++d) {
        pcg32_t b = pcg32_advanced(r, d);
        if (b.state != a.state || b.inc != a.inc) { printf("mismatch at %llu\n", d); return 1; }
        pcg32_next(&a);
    }
    pcg32_t far = pcg32_advanced(r, 2ull * 1920 * 1080 + 77);
    pcg32_t step = r;
    for (unsigned long long d = 0; d < 2ull * 1920 * 1080 + 77; ++d) pcg32_next(&step);
    if (far.state != step.state) { printf("far mismatch\n"); return 1; }
    printf("ok\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_pcg32_jump_ahead_equals_stepping(tmp_path):
    c = tmp_path / "t.c"
    c.write_text(SRC)
    exe = tmp_path / "t"
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "compactcnncascade_b200", "csrc"), "-o", str(exe), str(c)])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
