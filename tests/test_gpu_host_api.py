"""The C++ host mirror (qsm.rs_b200/host/qsm.hpp) compiled against libqsmgpu.so and run on
the GPU; its outputs are compared with the oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_host_api(tmp_path):
    exe = tmp_path / "host_api_test"
    lib = os.path.join(ROOT, "qsm.rs_b200", "lib")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "qsm.rs_b200", "host", "host_api_test.cpp"), "-L", lib, "-lqsmgpu",
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n = 16
    N = n ** 3
    res = np.fromfile(out, dtype=np.float64).reshape(9, N)
    grid = O.Grid.new(n, n, n)
    field = (0.01 * np.sin(0.7 * np.arange(N))).reshape(grid.shape)
    mask = np.ones(grid.shape, np.uint8)
    phase = 3.0 * np.sin(0.05 * np.arange(N))
    refs = [O.tkd(field, mask, grid, (0, 0, 1), O.TkdParams(0.15)),
            O.tv_admm(field, mask, grid, (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, 10)),
            O.laplacian_unwrap(phase.reshape(grid.shape), mask, grid),
            O.sharp(field, mask, grid, O.SharpParams(0.05, 3.0))[0],
            O.rts(field, mask, grid, (0, 0, 1), O.RtsParams(0.15, 1e5, 10.0, 0.0, 7, 4), exact_dc=True),
            O.nltv(field, mask, grid, (0, 0, 1), O.NltvParams(1e-3, 1.0, 0.0, 5, 2), exact_dc=True),
            O.ismv(field, mask, grid, O.IsmvParams(1e-6, 20, 3.0))[0],
            O.resharp(field, mask, grid, O.ResharpParams(3.0, 1e-4, 1e-6, 20))[0]]
    idx = np.arange(N, dtype=np.float64)
    tes = [0.005, 0.010, 0.015]
    ph3 = [0.3 + 150.0 * np.sin(0.01 * idx) * te + 0.01 * np.cos(3.0 * idx + te) for te in tes]
    mg3 = [1.0 + 0.5 * np.sin(0.2 * idx)] * 3
    fit = O.multi_echo_linear_fit(ph3, mg3, tes, mask.ravel(), True, 90.0)[0]
    assert np.array_equal(res[8], fit)
    for got, ref in zip(res, refs):
        ref = ref.ravel()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9
