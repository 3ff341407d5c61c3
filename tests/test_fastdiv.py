"""CPU check of the multiply-shift division the shared-memory FFT uses for its
Stockham index arithmetic (fast_div.h): exact for every divisor up to 20000
and every dividend below 2^24, in the host form and in the device form
(high word of (x << 8) * m, then shift)."""
import os
import subprocess

from oracle_lib import ROOT

SRC = r'''
#include <cstdio>
#include "fast_div.h"
using namespace at3r;
static unsigned dev_form(unsigned x, FastDiv d)
{
    return (unsigned)(((unsigned long long)(x << 8) * d.m) >> 32) >> d.l;
}
int main()
{
    long bad = 0;
    for (unsigned d = 1; d <= 20000; d++) {
        const FastDiv f = make_fast_div(d);
        for (unsigned long long k = 0; k * d < (1u << 24); k += (k < 2048 ? 1 : 211)) {
            for (int e = -1; e <= 1; e++) {
                const long long x = (long long)(k * d) + e;
                if (x < 0 || x >= (1 << 24)) continue;
                const unsigned want = (unsigned)(x / d);
                if (fast_div((unsigned)x, f) != want || dev_form((unsigned)x, f) != want) bad++;
            }
        }
        const unsigned top = (1u << 24) - 1;
        if (fast_div(top, f) != top / d || dev_form(top, f) != top / d) bad++;
    }
    std::printf("%ld\n", bad);
    return bad != 0;
}
'''


def test_fast_division_is_exact(tmp_path):
    src = tmp_path / "fastdiv.cpp"
    src.write_text(SRC)
    exe = tmp_path / "fastdiv"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "aretomo3_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "0", r.stdout + r.stderr
