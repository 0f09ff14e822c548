"""The TGV dipole stencil fit is host code in the library (no GPU needed): check the
C-ABI entry point against the oracle and the reference's own stencil tests."""
import numpy as np
import pytest

from oracle import qsm_oracle as O


@pytest.mark.parametrize("res,b0", [((1.0, 1.0, 1.0), (0.0, 0.0, 1.0)), ((1.0, 1.0, 2.0), (0.2, 0.3, 0.9)),
                                    ((0.8, 1.1, 1.5), (0.3, -0.2, 0.93))])
def test_oblique_stencil_matches_oracle(res, b0):
    from qsmgpu import inversion
    got = inversion.tgv_oblique_stencil(res, b0)
    want = O.tgv_oblique_stencil(res, b0)
    # same double-precision fit cast to float; the centre is a cancelling sum
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6)
    assert abs(float(got.astype(np.float64).sum())) < 1e-4  # src/inversion/tgv.rs:1452-1456
