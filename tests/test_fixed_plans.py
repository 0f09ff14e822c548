"""The compile-time FFT plan lists (QSM_FIXED_PLANS and QSM_FIXED_PLANS_WIDE in
csrc/fft_engine.cuh) must equal the host planner's output for each length, or
FixedPlan::matches never fires and the length silently takes the runtime engine.  The
planner (csrc/fft_plan.cpp) is compiled here with the host C++ compiler and asked for
every listed length."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "qsm.rs_b200", "csrc")

HARNESS = r"""
#include "fft_plan.h"
#include <cstdio>
#include <cstdlib>
int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    const int n = std::atoi(argv[a]);
    qsm::FftPlan1D pl;
    if (!qsm::make_fft_plan(n, &pl)) { std::printf("%d none\n", n); continue; }
    std::printf("%d %d", n, pl.T);
    for (int s = 0; s < pl.nstages; ++s) std::printf(" %d", pl.radix[s]);
    std::printf("\n");
  }
  return 0;
}
"""


def listed_plans():
    src = open(os.path.join(CSRC, "fft_engine.cuh")).read()
    out = {}
    for macro in ("QSM_FIXED_PLANS", "QSM_FIXED_PLANS_WIDE"):
        m = re.search(r"#define %s\(X\)(.*?)(?:\n\n|\n//)" % macro, src, re.S)
        assert m, macro
        body = m.group(1).replace("\\\n", " ")
        entries = re.findall(r"X\((\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)\)", body)
        assert entries, macro
        out[macro] = [tuple(int(v) for v in e) for e in entries]
    return out


def test_lists_are_disjoint_and_sorted():
    p = listed_plans()
    base = [e[0] for e in p["QSM_FIXED_PLANS"]]
    wide = [e[0] for e in p["QSM_FIXED_PLANS_WIDE"]]
    assert base == sorted(base) and wide == sorted(wide)
    assert not set(base) & set(wide)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_listed_plans_match_the_planner(tmp_path):
    harness = tmp_path / "plan_harness.cpp"
    harness.write_text(HARNESS)
    exe = tmp_path / "plan_harness"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", CSRC, str(harness), os.path.join(CSRC, "fft_plan.cpp"),
                    "-o", str(exe)], check=True)
    p = listed_plans()
    entries = p["QSM_FIXED_PLANS"] + p["QSM_FIXED_PLANS_WIDE"]
    res = subprocess.run([str(exe)] + [str(e[0]) for e in entries], check=True, capture_output=True, text=True)
    got = {}
    for line in res.stdout.split("\n"):
        if line.strip():
            f = line.split()
            got[int(f[0])] = f[1:]
    for n, t, r0, r1, r2 in entries:
        radices = [r0, r1] + ([r2] if r2 != 1 else [])
        assert got[n] == [str(t)] + [str(r) for r in radices], (n, got[n])
