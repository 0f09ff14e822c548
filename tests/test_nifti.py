"""NIfTI-1 I/O (src/io.rs:62-460): the host entry points of libqsmgpu.so, which need no
GPU, against the oracle's restatement and the reference's own tests (io.rs:457-872).
Writing is compared byte for byte; reading of every supported datatype, both byte
orders, scaling, 4D data and gzip is compared value for value."""
import gzip
import math
import os

import numpy as np
import pytest

from oracle import qsm_oracle as O
from qsmgpu import QsmError, DimensionMismatch
from qsmgpu import nifti as nf

IDENT = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]


def test_save_nifti_header_facts():
    """io.rs:478-500 and 679-723."""
    b = nf.save_nifti(np.zeros(8), (2, 2, 2), (1.0, 1.0, 1.0), IDENT)
    assert len(b) == 352 + 8 * 4 and b[344:348] == b"n+1\0"
    assert int.from_bytes(b[0:4], "little") == 348
    aff = [1.5, 0, 0, 5, 0, 2.5, 0, 10, 0, 0, 3.5, 15, 0, 0, 0, 1]
    b = nf.save_nifti(np.arange(1, 9.0), (2, 2, 2), (1.5, 2.5, 3.5), aff)
    a = np.frombuffer(b, "<i2", 8, 40)
    assert a[0] == 3 and a[1] == 2
    assert np.frombuffer(b, "<i2", 1, 70)[0] == 16 and np.frombuffer(b, "<i2", 1, 72)[0] == 32
    assert np.frombuffer(b, "<f4", 1, 108)[0] == 352.0 and np.frombuffer(b, "<f4", 1, 112)[0] == 1.0
    assert np.frombuffer(b, "<i2", 1, 254)[0] == 1
    assert abs(np.frombuffer(b, "<f4", 1, 80)[0] - 1.5) < 1e-6


@pytest.mark.parametrize("dims", [(2, 2, 2), (4, 4, 4), (7, 3, 5)])
def test_save_matches_oracle_bytes(dims):
    rng = np.random.default_rng(sum(dims))
    d = rng.normal(0, 100, int(np.prod(dims)))
    aff = [1.0, 0.1, 0.2, 10.0, 0.3, 2.0, 0.4, 20.0, 0.5, 0.6, 3.0, 30.0, 0, 0, 0, 1]
    assert nf.save_nifti(d, dims, (1.0, 2.0, 3.0), aff) == O.nifti_save_bytes(d, dims, (1.0, 2.0, 3.0), aff)


def test_data_values_and_roundtrips(tmp_path):
    """io.rs:503-620, 726-852: data values, file round trips (.nii and .nii.gz), affine."""
    data = [1.0, 2.0, -3.0, 4.5, 0.0, 100.0, -0.5, 999.0]
    b = nf.save_nifti(data, (2, 2, 2), (1, 1, 1), IDENT)
    assert np.allclose(np.frombuffer(b, "<f4", 8, 352), data)
    n = 64
    vals = np.arange(n) * 0.5 + 1.0
    aff = [1.0, 0, 0, 10.0, 0, 2.0, 0, 20.0, 0, 0, 3.0, 30.0, 0, 0, 0, 1]
    p = str(tmp_path / "rt.nii")
    nf.save_nifti_to_file(p, vals, (4, 4, 4), (1.0, 2.0, 3.0), aff)
    got = nf.read_nifti_file(p)
    assert got.dims == (4, 4, 4) and np.allclose(got.voxel_size, (1, 2, 3)) and np.abs(got.data - vals).max() < 0.01
    assert np.allclose(got.affine, aff, atol=0.01)
    pg = str(tmp_path / "rt.nii.gz")
    nf.save_nifti_to_file(pg, np.arange(n, dtype=float), (4, 4, 4), (1, 1, 1), IDENT)
    raw = open(pg, "rb").read()
    assert raw[:2] == b"\x1f\x8b"
    assert gzip.decompress(raw) == nf.save_nifti(np.arange(n, dtype=float), (4, 4, 4), (1, 1, 1), IDENT)
    assert np.array_equal(nf.read_nifti_file(pg).data, np.arange(n, dtype=float))
    assert nf.read_nifti_dims(pg) == (4, 4, 4) and nf.read_nifti_dims(p) == (4, 4, 4)
    f32 = (np.arange(n, dtype=np.float32) * np.float32(0.1)).astype(np.float64)
    nf.save_nifti_to_file(p, f32, (4, 4, 4), (1.5, 1.5, 1.5), IDENT)
    assert np.array_equal(nf.read_nifti_file(p).data, f32)
    big = np.sin(np.arange(512.0))
    ld = nf.load_nifti(nf.save_nifti(big, (8, 8, 8), (0.5, 0.5, 0.5), IDENT))
    assert ld.dims == (8, 8, 8) and np.abs(ld.data - big).max() < 0.01
    ld = nf.load_nifti(nf.save_nifti_gz(np.zeros(8), (2, 2, 2), (1, 1, 1), IDENT))
    assert ld.dims == (2, 2, 2)
    ld = nf.load_nifti(nf.save_nifti(np.ones(64), (4, 4, 4), (1, 1, 1), IDENT))
    assert ld.scl_slope == 1.0 and ld.scl_inter == 0.0


def test_errors(tmp_path):
    """io.rs:624-641 and 775-784: invalid bytes, corrupt gzip, missing file."""
    with pytest.raises(QsmError):
        nf.load_nifti(bytes(10))
    with pytest.raises(QsmError):
        nf.load_nifti(bytes([0x1F, 0x8B, 0, 0, 0]))
    with pytest.raises(QsmError) as e:
        nf.read_nifti_file(str(tmp_path / "nonexistent_file_12345.nii"))
    assert "Failed to read file" in str(e.value)
    hdr = bytearray(348)
    hdr[0:4] = (348).to_bytes(4, "little")
    hdr[344:348] = b"n+1\0"
    hdr[40:42] = (2).to_bytes(2, "little")
    with pytest.raises(QsmError) as e:
        nf.load_nifti(bytes(hdr) + bytes(4))
    assert "Expected at least 3D" in str(e.value)
    good = nf.save_nifti(np.ones(8), (2, 2, 2), (1, 1, 1), IDENT)
    with pytest.raises(QsmError):
        nf.load_nifti(good[:-4])  # voxels cut short


@pytest.mark.parametrize("dt", sorted(O.NIFTI_DTYPES))
@pytest.mark.parametrize("big", [False, True])
def test_load_every_datatype_matches_oracle(dt, big):
    rng = np.random.default_rng(dt)
    kind = np.dtype(O.NIFTI_DTYPES[dt])
    if kind.kind == "f":
        vals = rng.normal(0, 1e3, 60)
    else:
        info = np.iinfo(kind)
        vals = rng.integers(max(info.min, -2 ** 40), min(info.max, 2 ** 40), 60, endpoint=True)
    for slope, inter in [(0.0, 0.0), (0.5, -3.25), (1.0, 0.0), (2.5e-3, 7.0)]:
        raw = O.nifti_craft(vals, (3, 4, 5, 1), dt, big, slope, inter, (0.7, 0.8, 1.9))
        got = nf.load_nifti(raw)
        ref = O.nifti_load(raw)
        assert np.array_equal(got.data, ref["data"]), (dt, big, slope)
        assert got.dims == (3, 4, 5) and got.voxel_size == ref["voxel_size"]
        assert got.scl_slope == ref["scl_slope"] and got.scl_inter == ref["scl_inter"]
        assert np.array_equal(got.affine, ref["affine"])
        assert np.array_equal(nf.load_nifti(gzip.compress(raw)).data, ref["data"])


def test_4d_and_first_volume():
    """load_nifti takes the first volume of 4D data; load_nifti_4d all of them (io.rs:125-147, 195-221)."""
    vals = np.arange(3 * 4 * 5 * 4, dtype=np.float64) - 100.0
    aff = [0.9, 0, 0.1, -5, 0, 1.1, 0, -6, 0.2, 0, 1.3, -7]
    raw = O.nifti_craft(vals, (3, 4, 5, 4), 16, False, 0.0, 0.0, (0.9, 1.1, 1.3), sform=aff)
    one = nf.load_nifti(raw)
    assert one.dims == (3, 4, 5) and np.array_equal(one.data, vals[:60])
    assert np.allclose(one.affine, aff + [0, 0, 0, 1], atol=1e-6)
    data, dims4, vs, affine = nf.load_nifti_4d(raw)
    assert dims4 == (3, 4, 5, 4) and np.array_equal(data, vals)
    ref = O.nifti_load(raw, all_volumes=True)
    assert np.array_equal(data, ref["data"]) and np.array_equal(affine, ref["affine"])


def test_oracle_pinned_to_reference_layout():
    """The oracle's writer and reader agree with the reference's stated byte layout."""
    b = O.nifti_save_bytes(np.arange(8.0), (2, 2, 2), (1.5, 2.5, 3.5), IDENT)
    assert len(b) == 352 + 32 and b[344:348] == b"n+1\0" and b[348:352] == bytes(4)
    r = O.nifti_load(b)
    assert r["dims"] == (2, 2, 2, 1) and np.array_equal(r["data"], np.arange(8.0))
    assert r["scl_slope"] == 1.0 and math.isclose(r["voxel_size"][1], 2.5)
