"""On-disk arrays at the boundary (msgpu_read_array / msgpu_write_array /
msgpu_read_arrays / msgpu_read_arrays_start / msgpu_*_displacement): the
reference's 2-D array files (qc::ScalarArray<QC_2D>::save / load, bzip2 by
suffix) against files written by the reference's own savers, decoded bit for
bit as the reference's loader decodes them.  Host code only: no GPU needed."""
import gzip
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

IO = os.path.join(GOLDEN, "io")
FILES = ("ref_p9.q2bz", "ref_p8.dat.bz2", "ref_p5.pgm", "ref_pa.pgm", "ref_p2.pgm", "ref_p7.txt", "ref_p9.pgm",
         "dm_t6.dm3", "dm_t4.dm4", "dm_t2.dm3", "dm_t10.dm4")


@pytest.fixture(scope="module")
def io():
    import msgpu
    from msgpu import build
    build.build()
    return msgpu


@pytest.mark.parametrize("name", FILES)
def test_reads_reference_files_bit_exact(io, name):
    g = golden("io_expected.npz")
    a = io.read_array(os.path.join(IO, name))
    assert a.shape == g[name].shape == ((13, 21) if name.startswith("dm_") else (17, 33))
    assert np.array_equal(a, g[name])


@pytest.mark.parametrize("version", [3, 4])
@pytest.mark.parametrize("t", [2, 3, 4, 5, 6, 10])
def test_digital_micrograph_like_the_reference(io, tmp_path, version, t):
    """Every image type DM3Reader exports, in DM3 and DM4: the last image of
    the ImageList is read, other tags (groups, arrays of groups, strings) are
    skipped; decoded values as the reference's importer decodes them."""
    import msor
    from msgpu.dmfile import dm_bytes
    rng = np.random.default_rng(10 * version + t)
    a = rng.normal(0, 100, (11, 19)) + (200 if t in (4, 5, 10) else 0)
    if t in (4, 5, 10):
        a = np.clip(a, 0, 255)
    p = tmp_path / f"x.dm{version}"
    p.write_bytes(dm_bytes([(rng.normal(size=(4, 6)), 6), (a, t)], version))
    ours = io.read_array(str(p))
    assert ours.shape == (11, 19)
    assert np.array_equal(ours, np.asarray(a.astype({2: "<i2", 3: "<i4", 4: "<u2", 5: "<u4", 6: "<f4",
                                                      10: "<u1"}[t]), dtype=np.float64))
    if msor.have_ref():
        assert np.array_equal(msor.RefRunner().load_array(str(p)), ours)


def test_reads_reference_displacement(io):
    g = golden("io_expected.npz")
    phi = io.read_displacement(os.path.join(IO, "ref_deformation_04_%d.dat.bz2"), 17)
    assert np.array_equal(phi, g["deformation"])


@pytest.mark.parametrize("suffix,type_", [(".q2bz", 9), (".dat.bz2", 9), (".pgm", 9), (".gz", 9), (".q2bz", 8),
                                          (".zz", 8)])
def test_round_trip(io, tmp_path, suffix, type_):
    a = np.random.default_rng(5).normal(size=(9, 21)) * 1e3
    p = str(tmp_path / ("x" + suffix))
    io.write_array(p, a, type_)
    b = io.read_array(p)
    assert np.array_equal(b, a if type_ == 9 else a.astype(np.float32).astype(np.float64))


def test_reads_gzip_written_by_another_tool(io, tmp_path):
    a = np.arange(12.0).reshape(3, 4) - 5.5
    body = b"P9\n# from gzip\n4 3\n6\n" + a.tobytes()
    p = tmp_path / "g.gz"
    p.write_bytes(gzip.compress(body))
    assert np.array_equal(io.read_array(str(p)), a)


def test_reference_reads_our_files(io, tmp_path):
    import msor
    if not msor.have_ref():
        pytest.skip("the reference driver is not built here")
    r = msor.RefRunner()
    a = np.random.default_rng(6).normal(size=(17, 33))
    for name, t in (("o.q2bz", 9), ("o.dat.bz2", 8), ("o.pgm", 9)):
        p = str(tmp_path / name)
        io.write_array(p, a, t)
        assert np.array_equal(r.load_array(p), io.read_array(p))
    phi = np.random.default_rng(7).normal(size=(2, 17 * 17))
    mask = str(tmp_path / "ours_%d.dat.bz2")
    io.write_displacement(mask, phi, 17)
    assert np.array_equal(r.load_displacement(4, mask), phi)


def test_parallel_and_background_decoding(io, tmp_path):
    rng = np.random.default_rng(8)
    frames = rng.normal(size=(7, 33, 33))
    paths = []
    for i, f in enumerate(frames):
        p = str(tmp_path / f"f{i}.q2bz")
        io.write_array(p, f)
        paths.append(p)
    assert np.array_equal(io.read_arrays(paths, 33, 33, threads=3), frames)
    out = np.zeros((7, 33, 33))
    assert np.array_equal(io.ReadTask(paths, 33, 33, out, threads=4).wait(), frames)


def test_errors(io, tmp_path):
    with pytest.raises(io.MsgpuError, match="Could not open"):
        io.read_array(str(tmp_path / "missing.q2bz"))
    bad = tmp_path / "bad.q2bz"
    bad.write_bytes(b"BZh9 this is not bzip2")
    with pytest.raises(io.MsgpuError, match="bzip2"):
        io.read_array(str(bad))
    magic = tmp_path / "m.pgm"
    magic.write_bytes(b"P6\n1 1\n255\n\x00\x00\x00")
    with pytest.raises(io.MsgpuError, match="magic"):
        io.read_array(str(magic))
    trunc = tmp_path / "t.pgm"
    trunc.write_bytes(b"P9\n4 4\n1\n" + np.zeros(3).tobytes())
    with pytest.raises(io.MsgpuError, match="truncated"):
        io.read_array(str(trunc))
    p = str(tmp_path / "s.q2bz")
    io.write_array(p, np.zeros((5, 6)))
    with pytest.raises(io.MsgpuError, match="differs"):
        io.read_arrays([p], 5, 5)
    with pytest.raises(io.MsgpuError, match="%d"):
        io.read_displacement(str(tmp_path / "nomask.dat.bz2"), 5)
    out = np.zeros((1, 5, 5))
    with pytest.raises(io.MsgpuError, match="differs"):
        io.ReadTask([p], 5, 5, out).wait()
