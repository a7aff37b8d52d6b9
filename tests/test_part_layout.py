"""The part layout of the partitioned PCG (csrc/gpt_layout.h), compiled for the host and checked for
every horizon 2 .. 512 (no GPU): the parts and separators cover every knot exactly once, the
separators lie strictly between parts, the warps' work assignment (each part's knots, separator
s_j's residual rows by warp j) touches only existing knots, and the rows the factorisation reads
(the coupling after each walk) exist."""
import os
import subprocess

import pytest

from conftest import ROOT

PROGRAM = r"""
#include <cstdio>
#include "gpt_layout.h"
int main()
{
    for (int n = 2; n <= 512; ++n) {
        const gpt::QuadLayout L = gpt::quad_layout(n);
        if (L.P < 1 || L.P > gpt::QUAD_NWARP) return 1;
        int owner[512];
        for (int k = 0; k < n; ++k) owner[k] = 0;
        for (int p = 0; p < L.P; ++p)
            for (int k = L.a[p]; k <= L.b[p]; ++k) {
                if (k < 0 || k >= n) return 2;
                owner[k]++;
            }
        for (int j = 0; j < L.P - 1; ++j) {
            const int s = L.s[j];
            if (s < 1 || s >= n) return 3;
            owner[s]++;
            if (L.b[j] != s - 1 && !(L.b[j] < L.a[j] && L.a[j] == s)) return 4;  // part j ends at s_j - 1 (or is empty)
            if (L.a[j + 1] != s + 1) return 5;                                      // part j + 1 starts after s_j
        }
        for (int k = 0; k < n; ++k)
            if (owner[k] != 1) return 6;
        if (L.a[0] != 0 || L.b[L.P - 1] != n - 1) return 7;
        // the last part walks bottom-up from n - 1 toward s_{P-2}; its first row exists
        if (L.P >= 2 && L.a[L.P - 1] < 1) return 8;
        std::printf("%d %d %d %d %d\n", n, L.P, L.P > 1 ? L.s[0] : -1, L.P > 2 ? L.s[1] : -1, L.P > 3 ? L.s[2] : -1);
    }
    return 0;
}
"""


def test_partition_layout_covers_every_horizon(tmp_path):
    src = tmp_path / "layout.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "layout"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "gpu-pcg-tracking_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.returncode
    rows = {int(x.split()[0]): [int(v) for v in x.split()[1:]] for x in r.stdout.strip().split("\n")}
    assert rows[128][0] == 4 and rows[2][0] == 1 and rows[3][0] == 2
