"""CPU tests of the host-callable helpers of the device plan build (csrc/plan_build.cuh),
compiled as host code with nvcc and run here without a GPU.

The work-queue emission relies on three properties of them:
- the Schwarz-factor bucket is non-decreasing in Qabs, so a run sorted by bucket (descending)
  has its screened kets, by the bucket bound alone, as a suffix (bisection in unscreened_end);
- every Qabs lies below its bucket's upper bound, so that suffix is screened exactly;
- in a run so sorted, the bisection on the bucket bound plus a short scan back ends a bra's
  ket run exactly after its last unscreened ket (no unscreened quartet is left out);
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
    // the truncation of a bra's ket run: runs sorted as the plan sorts them (bucket descending,
    // any order within a bucket) end exactly after their last unscreened ket
    std::uniform_int_distribution<int> len(1, 400);
    std::uniform_real_distribution<double> lq(-25.0, 3.0), u01(0.0, 1.0);
    const double cuts[] = {1e-12, 5e-10, 1e-6, 1e-2};
    for (int trial = 0; trial < 4000; ++trial) {
        const int n = len(rng);
        std::vector<std::pair<int, double>> v(n);
        for (auto &e : v) {
            const double x = u01(rng) < 0.05 ? 0.0 : std::pow(10.0, lq(rng));
            e = {qabs_bucket(x), x};
        }
        std::shuffle(v.begin(), v.end(), rng);
        std::stable_sort(v.begin(), v.end(), [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
            return a.first > b.first;
        });
        std::vector<double2> bnd(n);
        for (int k = 0; k < n; ++k) bnd[k] = make_double2(v[k].second, 0.0);
        const int pb = std::uniform_int_distribution<int>(0, n - 1)(rng);
        const int kbeg = std::uniform_int_distribution<int>(0, pb)(rng);
        const int kend = trial % 2 ? pb + 1 : n;  // equal classes: kets up to the bra itself
        const double cut = cuts[trial % 4];
        int want = kbeg;
        for (int k = kbeg; k < kend; ++k)
            if (!(bnd[pb].x * bnd[k].x < cut)) want = k + 1;
        const int got = unscreened_end(bnd.data(), cut, pb, kbeg, kend);
        if (got != want) { ++bad; std::printf("run end %d, want %d (n %d)\n", got, want, n); }
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
