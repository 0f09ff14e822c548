"""NIfTI voxels straight to and from device memory (qsm_nifti_load_device /
qsm_nifti_save_device): the GPU decode of every stored datatype, byte order, scaling and
4D layout equals the host decoder bit for bit, and the GPU float32 encode gives the
host writer's bytes."""
import gzip

import numpy as np
import pytest
import torch

from oracle import qsm_oracle as O
from qsmgpu import nifti as nf

pytestmark = pytest.mark.gpu

IDENT = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]


@pytest.mark.parametrize("dt", sorted(O.NIFTI_DTYPES))
@pytest.mark.parametrize("big", [False, True])
def test_load_device_every_datatype(ctx64, dt, big):
    rng = np.random.default_rng(dt + big)
    kind = np.dtype(O.NIFTI_DTYPES[dt])
    n = 37 * 21 * 11
    if kind.kind == "f":
        vals = rng.normal(0, 1e3, n)
    else:
        info = np.iinfo(kind)
        vals = rng.integers(max(info.min, -2 ** 40), min(info.max, 2 ** 40), n, endpoint=True)
    for slope, inter in [(0.0, 0.0), (0.5, -3.25), (2.5e-3, 7.0)]:
        raw = O.nifti_craft(vals, (37, 21, 11, 1), dt, big, slope, inter)
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        for b in (raw, gzip.compress(raw)):
            h = nf.load_nifti_device(b, out.data_ptr(), n, ctx=ctx64)
            assert (h.nx, h.ny, h.nz) == (37, 21, 11)
            assert np.array_equal(out.cpu().numpy(), nf.load_nifti(raw).data), (dt, big, slope)


def test_load_device_4d_and_large():
    """All volumes of a 4D int16 image larger than one staging buffer (32 MB)."""
    import qsmgpu
    ctx = qsmgpu.Context(0, "f64")
    dims4 = (192, 160, 128, 4)
    n = int(np.prod(dims4))
    vals = (np.arange(n, dtype=np.int64) % 65521 - 32000).astype(np.int16)
    raw = O.nifti_craft(vals, dims4, 4, False, 0.25, 1.0)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    h = nf.load_nifti_device(raw, out.data_ptr(), n, all_volumes=True, ctx=ctx)
    assert h.nt == 4
    host, _, _, _ = nf.load_nifti_4d(raw)
    assert np.array_equal(out.cpu().numpy(), host)
    first = torch.empty(n // 4, dtype=torch.float64, device="cuda")
    nf.load_nifti_device(raw, first.data_ptr(), n // 4, ctx=ctx)
    assert np.array_equal(first.cpu().numpy(), host[: n // 4])
    with pytest.raises(qsmgpu.DimensionMismatch):
        nf.load_nifti_device(raw, first.data_ptr(), n // 4 + 1, ctx=ctx)


@pytest.mark.parametrize("dims", [(2, 2, 2), (64, 48, 40), (256, 256, 176)])
def test_save_device_matches_host(ctx64, dims):
    n = int(np.prod(dims))
    rng = np.random.default_rng(n)
    d = rng.normal(0, 0.1, n)
    aff = [1.0, 0.1, 0.2, 10.0, 0.3, 2.0, 0.4, 20.0, 0.5, 0.6, 3.0, 30.0, 0, 0, 0, 1]
    t = torch.from_numpy(d).cuda()
    host = nf.save_nifti(d, dims, (1.0, 1.1, 1.2), aff)
    assert nf.save_nifti_device(t.data_ptr(), dims, (1.0, 1.1, 1.2), aff, ctx=ctx64) == host
    gz = nf.save_nifti_device(t.data_ptr(), dims, (1.0, 1.1, 1.2), aff, gz=True, ctx=ctx64)
    assert gz[:2] == b"\x1f\x8b" and gzip.decompress(gz) == host
