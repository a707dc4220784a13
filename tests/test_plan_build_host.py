"""CPU tests of the host-callable helpers of the device plan build (csrc/plan_build.cuh),
compiled as host code with nvcc and run here without a GPU.

The work-queue emission relies on three properties of them:
- the Schwarz-factor bucket is non-decreasing in Qabs, so a run sorted by bucket (descending)
  has its screened kets, by the bucket bound alone, as a suffix (bisection in unscreened_end);
- every Qabs lies below its bucket's upper bound, so that suffix is screened exactly;
- a ket whose quartet with the bra needs no HGP lane split implies the same for every ket
  with fewer primitive pairs, so that in a run of descending counts a chunk that starts
  unsplit stays unsplit (splits above zero need not be monotone in the count: the walk tests
  every ket of a split chunk)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "molecularintegrals.jl_b200" / "csrc"

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include <algorithm>
#include "plan_build.cuh"
using namespace molints;

int main() {
    int bad = 0;
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> ex(-320.0, 300.0), fr(0.5, 1.0);
    std::vector<double> q = {0.0, 5e-324, 1e-310, 1e-300, 1e-30, 1.0, 1e30, 1e300, 1.7e308};
    for (int i = 0; i < 200000; ++i) q.push_back(fr(rng) * std::pow(10.0, ex(rng)));
    for (int e = -1074; e <= 1023; ++e) {  // every binary exponent and its neighbours
        const double x = std::ldexp(1.0, e);
        q.push_back(x);
        q.push_back(std::nextafter(x, 0.0));
        q.push_back(std::nextafter(x, HUGE_VAL));
    }
    std::sort(q.begin(), q.end());
    int prev = -1;
    for (double x : q) {
        const int b = qabs_bucket(x);
        if (b < 0 || b > 255) { ++bad; std::printf("bucket range %g -> %d\n", x, b); }
        if (b < prev) { ++bad; std::printf("not monotone at %g\n", x); }
        prev = b;
        const double hi = qabs_bucket_hi(b);
        if (x > 0.0 ? !(x < hi) : !(hi == 0.0)) { ++bad; std::printf("bound %g >= %g (b %d)\n", x, hi, b); }
    }
    // the lane split: pure and bounded; no split at nk means no split at every smaller nk
    for (double cost : {0.3, 1.0, 2.5, 9.0, 40.0})
        for (double lane : {20.0, 80.0, 320.0, 640.0, 1e6})
            for (int nb = 1; nb <= 64; ++nb) {
                bool split_below = false;
                for (int nk = 1; nk <= 64; ++nk) {
                    const int s = hgp_split(nb, nk, cost, lane), lg = s & 15, lgj = s >> 4;
                    if (lg > 5 || lgj > lg || (1 << lgj) > nk) { ++bad; std::printf("split %d %d\n", nb, nk); }
                    if (s != hgp_split(nb, nk, cost, lane)) ++bad;
                    if (lg == 0 && split_below) { ++bad; std::printf("unsplit above a split: nb %d nk %d\n", nb, nk); }
                    split_below = split_below || lg != 0;
                }
            }
    std::printf("%zu values, %d failures\n", q.size(), bad);
    return bad != 0;
}
"""


def test_bucket_and_split_properties(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    src = tmp_path / "plan_build_host.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "plan_build_host"
    # the headers' device code is compiled for the B200 as in the library; only host code runs
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
                        "--expt-relaxed-constexpr", "-I", str(CSRC), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout[-3000:]
    assert "0 failures" in run.stdout
