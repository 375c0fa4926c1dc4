"""The raw writer's JLD2 (HDF5) files: the lookup3 checksum against Jenkins' published test
vectors, the file's structure against the HDF5 format (user block, version-2 superblock and object
headers with valid checksums, compact groups, contiguous datasets) and the reference's dataset
names, shapes and column-major order (RawWriter.jl:19-56, Writer.jl:156-172), and exact round
trips."""
import struct

import numpy as np
import pytest

from epp import casegen, checkpoint, jld2


def test_lookup3_published_vectors():
    # the self-test values of Bob Jenkins' lookup3.c driver
    assert jld2.lookup3(b"") == 0xDEADBEEF
    assert jld2.lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert jld2.lookup3(b"Four score and seven years ago") == 0x17770551
    assert jld2.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def _raw_file(tmp_path, n=37, ni=6, nf=11):
    rng = np.random.default_rng(3)
    ip = rng.integers(-1000, 1000, size=(n, ni)).astype(np.int32)
    fp = rng.standard_normal((n, nf)).astype(np.float32)
    app = {"TMSTEP": 1234, "TimeValue": 0.125, "TimeStamp": "2026_12_04_06_30_00", "WriteStep": 5}
    path = str(tmp_path / "result_0005.jld2")
    jld2.write(path, {"appendix": app, "raw": {"int_properties": ip, "float_properties": fp}})
    return path, ip, fp, app


def test_round_trip_exact(tmp_path):
    path, ip, fp, app = _raw_file(tmp_path)
    d = jld2.read(path)
    assert set(d) == {"raw", "appendix"}
    assert list(d["appendix"]) == ["TMSTEP", "TimeValue", "TimeStamp", "WriteStep"]
    assert d["appendix"] == app
    assert d["raw"]["int_properties"].dtype == np.int32 and d["raw"]["float_properties"].dtype == np.float32
    assert np.array_equal(d["raw"]["int_properties"], ip)
    assert np.array_equal(d["raw"]["float_properties"], fp)


def test_file_structure(tmp_path):
    path, ip, fp, _ = _raw_file(tmp_path)
    buf = open(path, "rb").read()
    assert buf.startswith(b"HDF5-based Julia Data Format, version ")
    sb = buf[512:560]
    assert sb[:8] == b"\x89HDF\r\n\x1a\n" and sb[8] == 2 and sb[9] == 8 and sb[10] == 8
    base, ext, eof, root = struct.unpack_from("<QQQQ", sb, 12)
    assert base == 512 and ext == jld2.UNDEF and eof == len(buf) - 512
    assert struct.unpack_from("<I", sb, 44)[0] == jld2.lookup3(sb[:44])
    links = dict(jld2._links(jld2._parse_object_header(buf, base + root)))
    assert sorted(links) == ["appendix", "raw"]
    raw = dict(jld2._links(jld2._parse_object_header(buf, base + links["raw"])))
    for name, arr in (("int_properties", ip), ("float_properties", fp)):
        msgs = dict(jld2._parse_object_header(buf, base + raw[name]))
        space = msgs[jld2.MSG_DATASPACE]
        assert space[0] == 2 and space[1] == 2 and space[3] == 1
        # an n x m Julia matrix: HDF5 (C-order) dimensions (m, n), bytes in column-major order
        assert struct.unpack_from("<2Q", space, 4) == (arr.shape[1], arr.shape[0])
        layout = msgs[jld2.MSG_LAYOUT]
        assert layout[0] == 3 and layout[1] == 1
        addr, size = struct.unpack_from("<QQ", layout, 2)
        assert buf[base + addr:base + addr + size] == arr.tobytes(order="F")
        dt = msgs[jld2.MSG_DATATYPE]
        assert dt[0] & 0x0F == (0 if arr.dtype.kind == "i" else 1) and struct.unpack_from("<I", dt, 4)[0] == 4
    app = dict(jld2._links(jld2._parse_object_header(buf, base + links["appendix"])))
    assert list(app) == ["TMSTEP", "TimeValue", "TimeStamp", "WriteStep"]
    tm = dict(jld2._parse_object_header(buf, base + app["TMSTEP"]))
    assert tm[jld2.MSG_DATASPACE][3] == 0   # scalar
    assert struct.unpack_from("<I", tm[jld2.MSG_DATATYPE], 4)[0] == 8   # Int64


def test_corruption_detected(tmp_path):
    path, *_ = _raw_file(tmp_path)
    buf = bytearray(open(path, "rb").read())
    buf[512 + 48 + 10] ^= 0x40   # inside the root group's object header
    open(path, "wb").write(bytes(buf))
    with pytest.raises(jld2.FormatError):
        jld2.read(path)


def test_empty_rows_and_checkpoint_names(tmp_path):
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=8)
    ps = case.ps
    ps.is_alive[:] = 0
    path = checkpoint.save(ps, checkpoint.file_name(str(tmp_path), 0), checkpoint.appendix())
    assert path.endswith("result_0000.jld2")
    d = jld2.read(path)
    assert d["raw"]["int_properties"].shape == (0, ps.int_properties.shape[1])
    assert d["raw"]["float_properties"].shape == (0, ps.float_properties.shape[1])
