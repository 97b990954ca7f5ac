"""The invariant-divisor division the kernels decode site indices with
(FastDiv in csrc/lattice.cuh), compiled for the host with g++ from the same
header and checked against the hardware division: every divisor 1..2048 on
boundary and random dividends, and the lattice shapes of the workloads over
every site index.  CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "complb3d-lattice-boltzmann-fba-surrogate-cobrapy-glpk_b200", "csrc")

HARNESS = r"""
#include <cstdio>
#include <cstdint>
#include <random>
struct HostDim3 { unsigned x, y, z; };
static HostDim3 blockDim, threadIdx;     // the header's block helpers only need to compile here
#include "lattice.cuh"
using cl::FastDiv;
static int check(uint32_t d, uint32_t n) {
    FastDiv f; f.init(d);
    if (f.div(n) != n / d) { std::printf("FAIL d=%u n=%u got %u want %u\n", d, n, f.div(n), n / d); return 1; }
    return 0;
}
int main() {
    std::mt19937 rng(7);
    int bad = 0;
    for (uint32_t d = 1; d <= 2048 && !bad; ++d) {
        const uint32_t edge[] = {0u, 1u, d - 1, d, d + 1, 2 * d - 1, 2 * d, 0xffffffffu, 0xfffffffeu,
                                 0x80000000u, 0x7fffffffu, 0xffffffffu - d, (0xffffffffu / d) * d,
                                 (0xffffffffu / d) * d - 1};
        for (uint32_t n : edge) bad |= check(d, n);
        for (int k = 0; k < 20000; ++k) bad |= check(d, rng());
    }
    // every site index of the workloads' lattices: (n / nz, then / ny)
    const uint32_t shapes[][3] = {{512, 256, 256}, {256, 128, 128}, {128, 128, 128}, {26, 21, 17}, {22, 16, 16}};
    for (auto& s : shapes) {
        FastDiv fz, fy; fz.init(s[2]); fy.init(s[1]);
        const uint32_t N = s[0] * s[1] * s[2];
        for (uint32_t n = 0; n < N && !bad; ++n) {
            const uint32_t q = fz.div(n), x = fy.div(q);
            if (q != n / s[2] || x != q / s[1]) { std::printf("FAIL shape n=%u\n", n); bad = 1; }
        }
    }
    std::printf(bad ? "bad\n" : "ok\n");
    return bad;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_fastdiv_matches_division(tmp_path):
    src = tmp_path / "fastdiv.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "fastdiv"
    subprocess.run(["g++", "-O2", "-std=c++17", "-D__host__=", "-D__device__=", "-D__forceinline__=inline",
                    "-I" + CSRC, str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-500:]
