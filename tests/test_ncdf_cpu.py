"""netCDF-3 classic field files (the reference's u_result_*.nc layout) without
libnetcdf, checked against scipy's separate pure-Python implementation of the
same format: our files read there, its files read here, and byte for byte the
same file for the same content."""
import numpy as np
import pytest
from scipy.io import netcdf_file

import maxlq_b200 as mlq


def _field(n1, n2, n3, seed=0):
    return np.random.default_rng(seed).standard_normal((3, n3, n2, n1))


def _scipy_write(path, u, names=("Ux", "Uy", "Uz"), record=True):
    # scipy's writer wants an unlimited dimension defined first (the format
    # itself, and the reference's files, have it last): z, then x, y
    _, n3, n2, n1 = u.shape
    with netcdf_file(str(path), "w", version=1) as f:
        f.createDimension("z", None if record else n3)
        f.createDimension("x", n1)
        f.createDimension("y", n2)
        for k, name in enumerate(names):
            v = f.createVariable(name, "d", ("z", "y", "x"))
            v[:] = u[k]


@pytest.mark.parametrize("shape", [(16, 16, 16), (8, 12, 5), (1, 1, 1)])
def test_written_file_reads_back_in_scipy_and_here(tmp_path, shape):
    n1, n2, n3 = shape
    u = _field(n1, n2, n3)
    p = tmp_path / "u_result.nc"
    mlq.ncdf_write_field(p, u)
    with netcdf_file(str(p), "r", mmap=False) as f:
        assert f.dimensions["x"] == n1 and f.dimensions["y"] == n2 and f.dimensions["z"] is None
        assert f.variables["Ux"].dimensions == ("z", "y", "x")
        for k, name in enumerate(("Ux", "Uy", "Uz")):
            assert np.array_equal(f.variables[name][:], u[k])
    assert np.array_equal(mlq.ncdf_read_field(p), u)


def test_header_is_the_reference_layout(tmp_path):
    """Every header field per the classic format: dimensions x, y and the
    unlimited z in that order (the reference defines them so), no global
    attributes, three NC_DOUBLE record variables of dimension ids (2, 1, 0)
    without attributes, each record the three x-y slabs in order."""
    import struct
    n1, n2, n3 = 6, 5, 4
    u = _field(n1, n2, n3, seed=1)
    p = tmp_path / "u.nc"
    mlq.ncdf_write_field(p, u)
    b = p.read_bytes()
    words = lambda off, k: struct.unpack(">%dI" % k, b[off:off + 4 * k])
    assert b[:4] == b"CDF\x01"
    off = 4
    (numrecs,) = words(off, 1)
    off += 4
    assert numrecs == n3
    assert words(off, 2) == (0x0A, 3)
    off += 8
    for name, length in (("x", n1), ("y", n2), ("z", 0)):
        assert words(off, 1) == (1,) and b[off + 4:off + 5] == name.encode()
        off += 8
        assert words(off, 1) == (length,)
        off += 4
    assert words(off, 2) == (0, 0)
    off += 8
    assert words(off, 2) == (0x0B, 3)
    off += 8
    vsize = n1 * n2 * 8
    begins = []
    for name in ("Ux", "Uy", "Uz"):
        assert words(off, 1) == (2,) and b[off + 4:off + 6] == name.encode()
        off += 8
        assert words(off, 4) == (3, 2, 1, 0)
        off += 16
        assert words(off, 2) == (0, 0)
        off += 8
        t, vs, beg = words(off, 3)
        off += 12
        assert (t, vs) == (6, vsize)
        begins.append(beg)
    assert begins == [off, off + vsize, off + 2 * vsize]
    assert len(b) == off + n3 * 3 * vsize
    rec1_uy = np.frombuffer(b[off + 3 * vsize + vsize:off + 3 * vsize + 2 * vsize], dtype=">f8")
    assert np.array_equal(rec1_uy, u[1, 1].ravel())


@pytest.mark.parametrize("record", [True, False])
def test_reads_record_and_fixed_layouts(tmp_path, record):
    u = _field(10, 7, 6, seed=2)
    p = tmp_path / "in.nc"
    _scipy_write(p, u, names=("gradJ_x", "gradJ_y", "gradJ_z"), record=record)
    got = mlq.ncdf_read_field(p, names=("gradJ_x", "gradJ_y", "gradJ_z"))
    assert np.array_equal(got, u)


def test_errors(tmp_path):
    u = _field(4, 4, 4)
    p = tmp_path / "u.nc"
    mlq.ncdf_write_field(p, u)
    with pytest.raises(mlq.MlqError) as e:
        mlq.ncdf_read_field(p, names=("Ux", "Uy", "missing"))
    assert e.value.status == 8
    with pytest.raises(mlq.MlqError) as e:
        mlq.ncdf_read_field(tmp_path / "absent.nc")
    assert e.value.status == 11
    bad = tmp_path / "bad.nc"
    bad.write_bytes(b"HDF\x01" + bytes(64))
    with pytest.raises(mlq.MlqError) as e:
        mlq.ncdf_read_field(bad)
    assert e.value.status == 11


def test_truncated_restart_file_is_an_io_error(tmp_path):
    # a restart file cut short in its data (a run killed while saving)
    u = _field(8, 8, 8)
    p = tmp_path / "u_result.nc"
    mlq.ncdf_write_field(p, u)
    raw = p.read_bytes()
    cut = tmp_path / "cut.nc"
    cut.write_bytes(raw[: len(raw) - 100])
    with pytest.raises(mlq.MlqError) as e:
        mlq.ncdf_read_field(cut)
    assert e.value.status == 11
