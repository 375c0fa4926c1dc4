"""The reference's raw-writer files (JLD2, an HDF5 container) written and read without an HDF5
library.

The reference's `DataIO` raw writer stores, per output step, one JLD2 file holding the groups
`raw` (datasets `int_properties`, `float_properties`: the alive rows of the property matrices) and
`appendix` (scalars `TMSTEP`, `TimeValue`, `WriteStep` and the string `TimeStamp`)
(src/DataIO/Writer/RawWriter.jl:19-56, src/DataIO/Writer/Writer.jl:156-172), and `DataIO.load!`
reads them back by those names (Writer.jl:214-230).  This image has no HDF5 library, so this module
writes that file from the published HDF5 file-format specification (version-2 superblock and
object headers, compact link storage in the groups, contiguous datasets) behind the 512-byte user
block a JLD2 file starts with, and reads back exactly what it writes.  The reference writes its
datasets Zstd-compressed in chunks; these files are uncompressed and contiguous, which a JLD2 or
HDF5 reader reads the same way.

Julia arrays are column-major: an n x m matrix is stored as its column-major bytes with the
dataspace dimensions reversed, (m, n), as HDF5 records C-order dimensions.

Checksums of the superblock and the object headers are Bob Jenkins' lookup3 `hashlittle` with
seed 0, as the HDF5 format prescribes; the implementation is pinned on Jenkins' published test
vectors (tests/test_jld2.py).
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
USER_BLOCK = 512
JLD2_HEADER = b"HDF5-based Julia Data Format, version 0.1.1"
HDF5_SIGNATURE = b"\x89HDF\r\n\x1a\n"

# object header message types (HDF5 format specification, section IV.A.2)
MSG_DATASPACE = 0x01
MSG_LINK_INFO = 0x02
MSG_DATATYPE = 0x03
MSG_FILL_VALUE = 0x05
MSG_LINK = 0x06
MSG_LAYOUT = 0x08
MSG_GROUP_INFO = 0x0A

M32 = 0xFFFFFFFF


def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & M32


def lookup3(data, initval=0):
    """Bob Jenkins' lookup3 hashlittle over `data` (bytes), the checksum of HDF5 metadata."""
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & M32
    if n == 0:
        return c
    k = 0
    while n > 12:
        a = (a + int.from_bytes(data[k:k + 4], "little")) & M32
        b = (b + int.from_bytes(data[k + 4:k + 8], "little")) & M32
        c = (c + int.from_bytes(data[k + 8:k + 12], "little")) & M32
        # mix(a, b, c)
        a = (a - c) & M32; a ^= _rot(c, 4); c = (c + b) & M32
        b = (b - a) & M32; b ^= _rot(a, 6); a = (a + c) & M32
        c = (c - b) & M32; c ^= _rot(b, 8); b = (b + a) & M32
        a = (a - c) & M32; a ^= _rot(c, 16); c = (c + b) & M32
        b = (b - a) & M32; b ^= _rot(a, 19); a = (a + c) & M32
        c = (c - b) & M32; c ^= _rot(b, 4); b = (b + a) & M32
        k += 12
        n -= 12
    tail = bytes(data[k:k + n]) + b"\x00" * (12 - n)   # the last 1..12 bytes, zero-padded
    a = (a + int.from_bytes(tail[0:4], "little")) & M32
    b = (b + int.from_bytes(tail[4:8], "little")) & M32
    c = (c + int.from_bytes(tail[8:12], "little")) & M32
    # final(a, b, c)
    c ^= b; c = (c - _rot(b, 14)) & M32
    a ^= c; a = (a - _rot(c, 11)) & M32
    b ^= a; b = (b - _rot(a, 25)) & M32
    c ^= b; c = (c - _rot(b, 16)) & M32
    a ^= c; a = (a - _rot(c, 4)) & M32
    b ^= a; b = (b - _rot(a, 14)) & M32
    c ^= b; c = (c - _rot(b, 24)) & M32
    return c


# ---- datatype messages (format specification IV.A.2.d) ------------------------------------------
def _dt_fixed(size, signed=True):
    """Little-endian two's-complement integer of `size` bytes."""
    head = bytes([(1 << 4) | 0, 0x08 if signed else 0x00, 0, 0]) + struct.pack("<I", size)
    return head + struct.pack("<HH", 0, 8 * size)


def _dt_float(size):
    """Little-endian IEEE 754 binary32 or binary64 (implied leading mantissa bit)."""
    if size == 4:
        sign, exp_loc, exp_size, mant_size, bias = 31, 23, 8, 23, 127
    elif size == 8:
        sign, exp_loc, exp_size, mant_size, bias = 63, 52, 11, 52, 1023
    else:
        raise ValueError("float of %d bytes" % size)
    head = bytes([(1 << 4) | 1, 0x20, sign, 0]) + struct.pack("<I", size)
    return head + struct.pack("<HHBBBBI", 0, 8 * size, exp_loc, exp_size, 0, mant_size, bias)


def _dt_string(size):
    """Fixed-length ASCII string of `size` bytes, null-padded."""
    return bytes([(1 << 4) | 3, 0x01, 0, 0]) + struct.pack("<I", size)


def _datatype_of(arr):
    k, size = arr.dtype.kind, arr.dtype.itemsize
    if k == "i":
        return _dt_fixed(size, True)
    if k == "u":
        return _dt_fixed(size, False)
    if k == "f":
        return _dt_float(size)
    if k == "S":
        return _dt_string(size)
    raise TypeError("no HDF5 datatype for %s" % arr.dtype)


# ---- object headers (version 2, "OHDR") ----------------------------------------------------------
def _message(mtype, body, flags=0):
    return struct.pack("<BHB", mtype, len(body), flags) + body


def _object_header(messages):
    """A version-2 object header holding `messages` (encoded by _message) in its only chunk."""
    body = b"".join(messages)
    n = len(body)
    if n < 1 << 8:
        size_flag, size_field = 0, struct.pack("<B", n)
    elif n < 1 << 16:
        size_flag, size_field = 1, struct.pack("<H", n)
    else:
        size_flag, size_field = 2, struct.pack("<I", n)
    head = b"OHDR" + bytes([2, size_flag]) + size_field
    blob = head + body
    return blob + struct.pack("<I", lookup3(blob))


def _group_messages(links):
    """Link info, group info and one link message per (name, address): compact link storage."""
    msgs = [_message(MSG_LINK_INFO, struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF)),
            _message(MSG_GROUP_INFO, struct.pack("<BB", 0, 0))]
    for name, addr in links:
        nb = name.encode("ascii")
        if not 0 < len(nb) < 256:
            raise ValueError("link name %r" % name)
        msgs.append(_message(MSG_LINK, struct.pack("<BBB", 1, 0, len(nb)) + nb + struct.pack("<Q", addr)))
    return msgs


def _dataset_messages(arr, data_addr):
    """Dataspace (scalar or simple, dimensions reversed for column-major data), datatype, fill value
    (allocated late, never written) and a contiguous layout at `data_addr`."""
    if arr.ndim == 0:
        space = struct.pack("<BBBB", 2, 0, 0, 0)
    else:
        dims = arr.shape[::-1]
        space = struct.pack("<BBBB", 2, len(dims), 0, 1) + b"".join(struct.pack("<Q", d) for d in dims)
    fill = struct.pack("<BB", 3, 0x02 | (1 << 2))
    layout = struct.pack("<BBQQ", 3, 1, data_addr if arr.nbytes else UNDEF, arr.nbytes)
    return [_message(MSG_DATASPACE, space), _message(MSG_DATATYPE, _datatype_of(arr), flags=0x01),
            _message(MSG_FILL_VALUE, fill, flags=0x01), _message(MSG_LAYOUT, layout)]


def _column_major_bytes(arr):
    return np.asarray(arr).tobytes(order="F")


def _as_dataset(v):
    """A Python or NumPy value as the array written for it (Julia's Int64, Float64, String for
    Python scalars, as the reference's appendix holds them)."""
    if isinstance(v, str):
        b = v.encode("ascii")
        return np.array(b if b else b"\x00", dtype="S%d" % max(len(b), 1))
    if isinstance(v, (bool, np.bool_)):
        raise TypeError("no Bool datasets in the raw writer")
    if isinstance(v, (int, np.integer)) and not isinstance(v, np.ndarray):
        return np.array(v, dtype=np.int64)
    if isinstance(v, (float, np.floating)) and not isinstance(v, np.ndarray):
        return np.array(v, dtype=np.float64)
    return np.asarray(v)


def write(path, groups):
    """Write `groups` ({group: {dataset: value}}, in order) as a JLD2 file at `path`."""
    groups = {g: {k: _as_dataset(v) for k, v in ds.items()} for g, ds in groups.items()}
    # sizes first: an address is 8 bytes whatever its value, so every header's size is known
    pos = 48   # the superblock
    root_addr = pos
    pos += len(_object_header(_group_messages([(g, 0) for g in groups])))
    g_addr, d_addr = {}, {}
    for g, ds in groups.items():
        g_addr[g] = pos
        pos += len(_object_header(_group_messages([(k, 0) for k in ds])))
        for k, arr in ds.items():
            d_addr[g, k] = pos
            pos += len(_object_header(_dataset_messages(arr, 0)))
    data_addr = {}
    for g, ds in groups.items():
        for k, arr in ds.items():
            pos = (pos + 7) & ~7
            data_addr[g, k] = pos
            pos += arr.nbytes
    eof = pos
    out = bytearray(eof)
    sb = HDF5_SIGNATURE + bytes([2, 8, 8, 0]) + struct.pack("<QQQQ", USER_BLOCK, UNDEF, eof, root_addr)
    out[0:48] = sb + struct.pack("<I", lookup3(sb))

    def put(addr, blob):
        out[addr:addr + len(blob)] = blob

    put(root_addr, _object_header(_group_messages([(g, g_addr[g]) for g in groups])))
    for g, ds in groups.items():
        put(g_addr[g], _object_header(_group_messages([(k, d_addr[g, k]) for k in ds])))
        for k, arr in ds.items():
            put(d_addr[g, k], _object_header(_dataset_messages(arr, data_addr[g, k])))
            put(data_addr[g, k], _column_major_bytes(arr))
    header = JLD2_HEADER + b"\x00"
    with open(path, "wb") as f:
        f.write(header + b"\x00" * (USER_BLOCK - len(header)))
        f.write(bytes(out))
    return path


# ---- reading ---------------------------------------------------------------------------------------
class FormatError(ValueError):
    pass


def _parse_object_header(buf, at):
    """The (type, body) messages of the version-2 object header at absolute offset `at`, after
    checking its signature and checksum."""
    if buf[at:at + 4] != b"OHDR" or buf[at + 4] != 2:
        raise FormatError("no version-2 object header at %d" % at)
    flags = buf[at + 5]
    p = at + 6
    if flags & 0x20:   # access, modification, change and birth times
        p += 16
    if flags & 0x10:   # attribute storage phase change values
        p += 4
    width = 1 << (flags & 3)
    n = int.from_bytes(buf[p:p + width], "little")
    p += width
    end = p + n
    if struct.unpack_from("<I", buf, end)[0] != lookup3(bytes(buf[at:end])):
        raise FormatError("object header checksum mismatch at %d" % at)
    msgs = []
    extra = 2 if flags & 0x04 else 0   # creation order of each message
    while end - p >= 4 + extra:
        mtype, size, _mflags = struct.unpack_from("<BHB", buf, p)
        p += 4 + extra
        msgs.append((mtype, bytes(buf[p:p + size])))
        p += size
    for mtype, _ in msgs:
        if mtype == 0x10:
            raise FormatError("object header continuation blocks are not supported")
    return msgs


def _links(msgs):
    out = []
    for mtype, b in msgs:
        if mtype != MSG_LINK:
            continue
        if b[0] != 1:
            raise FormatError("link message version %d" % b[0])
        flags, p = b[1], 2
        ltype = 0
        if flags & 0x08:
            ltype = b[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        width = 1 << (flags & 3)
        ln = int.from_bytes(b[p:p + width], "little")
        p += width
        name = b[p:p + ln].decode("utf-8")
        p += ln
        if ltype != 0:
            raise FormatError("link %r is not a hard link" % name)
        out.append((name, struct.unpack_from("<Q", b, p)[0]))
    return out


def _dtype(b):
    cls, size = b[0] & 0x0F, struct.unpack_from("<I", b, 4)[0]
    if cls in (0, 1) and b[1] & 0x01:
        raise FormatError("big-endian data")
    if cls == 0:
        return np.dtype("<%s%d" % ("i" if b[1] & 0x08 else "u", size))
    if cls == 1:
        return np.dtype("<f%d" % size)
    if cls == 3:
        return np.dtype("S%d" % size)
    raise FormatError("datatype class %d" % cls)


def _dataset(buf, base, msgs):
    dims, dt, data = None, None, None
    for mtype, b in msgs:
        if mtype == MSG_DATASPACE:
            if b[0] == 2:
                nd, flags, kind = b[1], b[2], b[3]
                dims = () if kind == 0 else tuple(struct.unpack_from("<%dQ" % nd, b, 4))
            elif b[0] == 1:
                nd = b[1]
                dims = tuple(struct.unpack_from("<%dQ" % nd, b, 8))
            else:
                raise FormatError("dataspace version %d" % b[0])
        elif mtype == MSG_DATATYPE:
            dt = _dtype(b)
        elif mtype == MSG_LAYOUT:
            if b[0] != 3:
                raise FormatError("layout version %d" % b[0])
            if b[1] == 0:
                size = struct.unpack_from("<H", b, 2)[0]
                data = b[4:4 + size]
            elif b[1] == 1:
                addr, size = struct.unpack_from("<QQ", b, 2)
                data = b"" if addr == UNDEF else bytes(buf[base + addr:base + addr + size])
            else:
                raise FormatError("chunked layout (compressed datasets) is not supported")
    if dims is None or dt is None or data is None:
        raise FormatError("dataset without dataspace, datatype or layout")
    arr = np.frombuffer(data, dtype=dt, count=int(np.prod(dims)) if dims else 1)
    if dims == ():
        v = arr[0]
        return v.rstrip(b"\x00").decode("ascii") if dt.kind == "S" else v.item()
    return arr.reshape(dims).T.copy()   # C-order dimensions reversed: the Julia (column-major) shape


def read(path):
    """{group: {dataset: value}} of a file `write` produced (or any HDF5 file of the same forms:
    version-2/3 superblock, version-2 object headers, compact groups, contiguous or compact data)."""
    with open(path, "rb") as f:
        buf = f.read()
    at = 0
    while at < len(buf) and buf[at:at + 8] != HDF5_SIGNATURE:
        at = USER_BLOCK if at == 0 else 2 * at
    if at >= len(buf):
        raise FormatError("no HDF5 superblock in %s" % path)
    if buf[at + 8] not in (2, 3) or buf[at + 9] != 8 or buf[at + 10] != 8:
        raise FormatError("superblock version %d with %d-byte offsets" % (buf[at + 8], buf[at + 9]))
    base, _ext, _eof, root = struct.unpack_from("<QQQQ", buf, at + 12)
    if struct.unpack_from("<I", buf, at + 44)[0] != lookup3(bytes(buf[at:at + 44])):
        raise FormatError("superblock checksum mismatch")
    out = {}
    for g, ga in _links(_parse_object_header(buf, base + root)):
        gm = _parse_object_header(buf, base + ga)
        if any(t == MSG_LINK_INFO for t, _ in gm):
            out[g] = {k: _dataset(buf, base, _parse_object_header(buf, base + a)) for k, a in _links(gm)}
        else:
            out[g] = _dataset(buf, base, gm)
    return out
