"""GPU test of qsm_tkd_device_noalloc, the TKD entry point that allocates no device
memory (its scratch is an array in the library's own device memory).  It exists for
callers that cannot call cudaMalloc — for example when another framework's caching
allocator has reserved the GPU, or inside a real-time loop that must not trigger the
device synchronisation of an allocation.

The result must match the regular entry point (qsm_tkd_device, f64 context) within
the f64 closed-form tolerance used by the other parity tests (1e-10 relative L2), on
two calls in a row with different inputs, so that stale scratch from the first call
cannot go unnoticed.  The file is named to be collected last.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tkd_noalloc_matches_tkd_device():
    import torch
    import qsmgpu
    from qsmgpu import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nx, ny, nz = 48, 40, 36
    grid = _lib.QsmGrid(nx, ny, nz, 1.0, 0.9, 1.1)
    bdir = (C.c_double * 3)(math.sin(0.3), 0.1, math.cos(0.3))
    params = _lib.QsmTkdParams(0.19)
    rng = np.random.default_rng(11)
    mask = torch.from_numpy((rng.random(nx * ny * nz) > 0.15).astype(np.uint8)).to(dev)
    ctx = qsmgpu.Context(0, "f64")
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        field = torch.from_numpy(rng.standard_normal(nx * ny * nz) * 0.05).to(dev)
        out_ref = torch.empty_like(field)
        out_na = torch.full_like(field, float("nan"))
        torch.cuda.synchronize()
        st = lib.qsm_tkd_device(ctx.handle, C.c_void_p(field.data_ptr()), C.c_void_p(mask.data_ptr()),
                                C.byref(grid), C.cast(bdir, _lib.c_double_p), C.byref(params),
                                C.c_void_p(out_ref.data_ptr()))
        assert st == 0, ctx.last_error()
        st = lib.qsm_tkd_device_noalloc(C.c_void_p(field.data_ptr()), C.c_void_p(mask.data_ptr()), C.byref(grid),
                                        C.cast(bdir, _lib.c_double_p), C.byref(params),
                                        C.c_void_p(out_na.data_ptr()), C.c_void_p(stream))
        assert st == 0, f"call {call}: status {st}"
        torch.cuda.synchronize()
        a = out_na.cpu().numpy()
        b = out_ref.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert _rel(a, b) < 1e-10, f"call {call}: rel-L2 {_rel(a, b):.3e}"
        assert np.all(a[mask.cpu().numpy() == 0] == 0.0)
    ctx.close()


def test_tkd_noalloc_rejects_oversized_volume():
    import torch
    from qsmgpu import _lib

    lib = _lib.load()
    torch.cuda.set_device(0)
    big = _lib.QsmGrid(256, 256, 256, 1.0, 1.0, 1.0)  # scratch needs ~0.27 GB > 48 MiB
    bdir = (C.c_double * 3)(0.0, 0.0, 1.0)
    params = _lib.QsmTkdParams(0.15)
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    st = lib.qsm_tkd_device_noalloc(C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), C.byref(big),
                                    C.cast(bdir, _lib.c_double_p), C.byref(params), C.c_void_p(dummy.data_ptr()),
                                    None)
    assert st == 3  # QSM_ERR_UNSUPPORTED_SIZE, before any kernel runs
