"""CPU checks of the C ABI boundary: the library loads and exports every symbol that
include/qsmgpu.h declares.  Nothing here launches a kernel."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qsmgpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qsm_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from qsmgpu import _lib
    return _lib.load()


def test_header_declares_functions():
    names = declared_functions()
    assert "qsm_tv_admm" in names and "qsm_run_dipole_inversion" in names and len(names) > 30


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_library_exports_only_the_abi():
    from qsmgpu import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    qsm = {s for s in exported if s.startswith("qsm_")}
    assert qsm == set(declared_functions())


def test_python_binding_covers_header():
    from qsmgpu import _lib
    assert set(_lib.EXPORTED_SYMBOLS) == set(declared_functions())


def test_host_only_entry_points(lib):
    from qsmgpu import _lib
    assert b"sm_100a" in lib.qsm_version()
    p = _lib.QsmTvParams()
    lib.qsm_tv_params_default(C.byref(p))
    assert (p.lambda_, p.rho, p.tol, p.max_iter) == (2e-4, 2e-2, 1e-3, 250)  # src/inversion/tv.rs:34-42
    v = _lib.QsmVsharpParams()
    lib.qsm_vsharp_params_default(C.byref(v))
    assert (v.threshold, v.max_radius, v.min_radius) == (0.05, 12.0, 1.0)
    s = _lib.QsmSharpParams()
    lib.qsm_sharp_params_default(C.byref(s))
    assert (s.threshold, s.radius) == (0.05, 6.0)
    t = _lib.QsmTkdParams()
    lib.qsm_tkd_params_default(C.byref(t))
    assert t.threshold == 0.15
    k = _lib.QsmTikhonovParams()
    lib.qsm_tikhonov_params_default(C.byref(k))
    assert (k.lambda_, k.reg) == (0.01, 0)
    il = _lib.QsmIlsqrParams()
    lib.qsm_ilsqr_params_default(C.byref(il))
    assert (il.tol, il.max_iter) == (0.01, 50)  # src/inversion/ilsqr.rs:27-34
    ic = _lib.QsmInversionConfig()
    lib.qsm_inversion_config_default(C.byref(ic))
    assert ic.algorithm == 4  # Rts, src/pipeline/config.rs:251
    assert (ic.ilsqr.tol, ic.ilsqr.max_iter) == (0.01, 50)
    assert (ic.rts.delta, ic.rts.mu, ic.rts.rho, ic.rts.tol, ic.rts.max_iter, ic.rts.lsmr_iter) == \
        (0.15, 1e5, 10.0, 1e-2, 20, 4)  # src/inversion/rts.rs:40-51
    assert (ic.nltv.lambda_, ic.nltv.mu, ic.nltv.tol, ic.nltv.max_iter, ic.nltv.newton_iter) == \
        (1e-3, 1.0, 1e-3, 250, 10)  # src/inversion/nltv.rs:38-48
    bc = _lib.QsmBgRemovalConfig()
    lib.qsm_bg_removal_config_default(C.byref(bc))
    assert bc.algorithm == 0  # Vsharp


def test_grid_support_planner(lib):
    from qsmgpu import _lib
    ok = lambda *d: lib.qsm_grid_supported(C.byref(_lib.QsmGrid(*d, 1.0, 1.0, 1.0)))
    assert ok(256, 256, 176) and ok(64, 64, 64) and ok(384, 384, 256) and ok(225, 135, 125)
    assert ok(1, 7, 13) and ok(2, 3, 11)
    # prime factors above 13 take Bluestein plans up to 2048 (MNI 182x218x182: 218 = 2*109)
    assert ok(17, 8, 8) and ok(8, 8, 19) and ok(182, 218, 182) and ok(2039, 23, 127) and ok(2048, 4096, 1)
    assert not ok(2053, 8, 8) and not ok(8, 4097, 8) and not ok(8, 8, 8192) and not ok(8, 8, 4094)


def test_null_context_rejected(lib):
    assert lib.qsm_ctx_destroy(None) == 1
    assert lib.qsm_tv_admm(None, None, None, None, None, None, _progress_none(), None, None) == 1


def _progress_none():
    from qsmgpu import _lib
    return _lib.PROGRESS_FN()
