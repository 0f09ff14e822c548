"""GPU parity of the multi-echo fits (src/utils/multi_echo.rs:450-804) against the
float64 oracle.  The kernels evaluate the reference's per-voxel sums in its order with
explicitly rounded double operations, so field, offset, residual and B0 are compared
bit for bit, and the reliability mask (a threshold at an exact order statistic of the
residuals) must match exactly."""
import math

import numpy as np
import pytest

from qsmgpu import multi_echo as me
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu


def echo_case(n, tes, seed, zero_mag_frac=0.05, mask_frac=0.8):
    rng = np.random.default_rng(seed)
    slope = rng.normal(0, 150.0, n)
    offset = rng.normal(0, 0.3, n)
    ph = [offset + slope * te + rng.normal(0, 0.05, n) for te in tes]
    mags = [np.abs(rng.normal(1.0, 0.3, n)) * math.exp(-te / 0.04) for te in tes]
    z = rng.random(n) < zero_mag_frac
    for m in mags:
        m[z] = 0.0
    mask = (rng.random(n) < mask_frac).astype(np.uint8)
    return ph, mags, mask


TES = [[0.004, 0.012, 0.020, 0.028], [0.005, 0.010, 0.015], [0.003, 0.008, 0.013, 0.018, 0.023]]


@pytest.mark.parametrize("tes", TES, ids=["4echo", "3echo", "5echo"])
def test_b0_weighted_bit_exact(ctx64, tes):
    ph, mags, mask = echo_case(50_000, tes, len(tes))
    for wt in range(5):
        got = me.calculate_b0_weighted(ph, mags, tes, mask, wt, ctx=ctx64)
        ref = O.calculate_b0_weighted(ph, mags, tes, mask, wt)
        assert np.array_equal(got, ref), (wt, np.abs(got - ref).max())


@pytest.mark.parametrize("tes", TES, ids=["4echo", "3echo", "5echo"])
@pytest.mark.parametrize("offset", [True, False])
@pytest.mark.parametrize("pct", [0.0, 50.0, 90.0, 100.0])
def test_linear_fit_bit_exact(ctx64, tes, offset, pct):
    ph, mags, mask = echo_case(60_000, tes, 7 + len(tes))
    got = me.multi_echo_linear_fit(ph, mags, tes, mask, offset, pct, ctx=ctx64)
    f, o, r, rm = O.multi_echo_linear_fit(ph, mags, tes, mask, offset, pct)
    assert np.array_equal(got.field, f)
    assert np.array_equal(got.phase_offset, o)
    assert np.array_equal(got.fit_residual, r)
    assert np.array_equal(got.reliability_mask, rm)
    if pct > 0:
        assert 0 < got.reliability_mask.sum() < mask.sum()


def test_linear_fit_mixed_context_is_float64(ctx32):
    """The fits always run in float64: the mixed context gives the same bits."""
    tes = TES[0]
    ph, mags, mask = echo_case(20_000, tes, 3)
    got = me.multi_echo_linear_fit(ph, mags, tes, mask, True, 90.0, ctx=ctx32)
    f, o, r, rm = O.multi_echo_linear_fit(ph, mags, tes, mask, True, 90.0)
    assert np.array_equal(got.field, f) and np.array_equal(got.reliability_mask, rm)


def test_reference_tests_on_gpu(ctx64):
    """src/utils/multi_echo.rs:1153-1491 through the GPU entry points."""
    tes = [0.005, 0.010, 0.015]
    ones = lambda n: np.ones(n, np.uint8)
    for wt in range(5):
        b0 = me.calculate_b0_weighted([np.full(16, 100.0 * te) for te in tes], [np.full(16, 2.0)] * 3, tes, ones(16),
                                      wt, ctx=ctx64)
        assert np.all(np.abs(b0 - 100.0 / (2 * math.pi)) < 1e-8)
    b0 = me.calculate_b0_weighted([np.full(4, 0.2 * te) for te in tes], [np.zeros(4)] * 3, tes, ones(4), ctx=ctx64)
    assert np.all(b0 == 0.0)
    r = me.multi_echo_linear_fit([np.full(32, 100.0 * te) for te in tes], [np.ones(32)] * 3, tes, ones(32), False,
                                 0.0, ctx=ctx64)
    assert np.all(np.abs(r.field - 100) < 1e-6) and np.all(r.phase_offset == 0) and np.all(r.reliability_mask == 1)
    tes4 = [0.005, 0.010, 0.015, 0.020]
    r = me.multi_echo_linear_fit([np.full(16, 0.5 + 200.0 * te) for te in tes4], [np.ones(16)] * 4, tes4, ones(16),
                                 True, 0.0, ctx=ctx64)
    assert np.all(np.abs(r.field - 200) < 1e-4) and np.all(np.abs(r.phase_offset - 0.5) < 1e-4)
    ph = [np.full(100, 100.0 * te) for te in tes]
    for e in range(3):
        ph[e][90:] += 2.0 if e % 2 == 0 else -2.0
    r = me.multi_echo_linear_fit(ph, [np.ones(100)] * 3, tes, ones(100), False, 80.0, ctx=ctx64)
    assert r.fit_residual[:90].max() < r.fit_residual[90:].min()
    ref = O.multi_echo_linear_fit(ph, [np.ones(100)] * 3, tes, ones(100), False, 80.0)
    assert np.array_equal(r.reliability_mask, ref[3])
    # all residuals exactly zero: the mask itself (values kept, multi_echo.rs:783-785)
    m5 = np.array([1, 2, 0, 1, 3], np.uint8)
    r = me.multi_echo_linear_fit([np.zeros(5)] * 3, [np.ones(5)] * 3, tes, m5, False, 50.0, ctx=ctx64)
    assert np.all(r.fit_residual == 0.0) and np.array_equal(r.reliability_mask, m5)
    # tiny nonzero roundoff residuals do count (as in the reference)
    ph = [np.full(5, 10.0 * te) for te in tes]
    r = me.multi_echo_linear_fit(ph, [np.ones(5)] * 3, tes, ones(5), False, 50.0, ctx=ctx64)
    assert np.array_equal(r.reliability_mask, O.multi_echo_linear_fit(ph, [np.ones(5)] * 3, tes, ones(5), False,
                                                                      50.0)[3])


def test_config_sizes_property(ctx64):
    """384x384x256, 4 echoes (the multi-echo benchmark shape): exact on a strided sample
    of voxels, and the reliability fraction sits at the percentile."""
    n = 384 * 384 * 256
    tes = TES[0]
    ph, mags, mask = echo_case(n, tes, 11, mask_frac=0.6)
    got = me.multi_echo_linear_fit(ph, mags, tes, mask, True, 90.0, ctx=ctx64)
    idx = np.arange(0, n, 997)
    f, o, r, _ = O.multi_echo_linear_fit([p[idx] for p in ph], [m[idx] for m in mags], tes, mask[idx], True, 0.0)
    assert np.array_equal(got.field[idx], f) and np.array_equal(got.fit_residual[idx], r)
    sel = (mask > 0) & (got.fit_residual > 0) & np.isfinite(got.fit_residual)
    k = int(0.9 * sel.sum())  # the threshold is the k-th smallest selected residual
    thr = np.partition(got.fit_residual[sel], k)[k]
    assert got.reliability_mask[sel].sum() == (got.fit_residual[sel] < thr).sum()
    assert np.array_equal(got.reliability_mask, ((mask > 0) & (got.fit_residual < thr)).astype(np.uint8))
