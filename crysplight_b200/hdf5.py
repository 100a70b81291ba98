"""A minimal HDF5 writer (and reader) for the output files, written from the
HDF5 File Format Specification (version 3.0), because no HDF5 library is
available to this package.

The files hold one root group with contiguous datasets and root attributes,
the structures the reference writes with HDF5.jl (src/output.jl:10-32,
scripts/shoot_gammas.jl:60-78):

  * superblock version 2 (offsets and lengths of 8 bytes, Jenkins lookup3
    checksum), root group object header version 2 with compact link storage
    (Link Info, Group Info and one hard-link Link message per dataset) and
    one Attribute message (version 3) per attribute;
  * each dataset: object header version 2 with Dataspace (version 2),
    Datatype (version 1: little-endian fixed-point, IEEE float or fixed-length
    null-terminated UTF-8 string), Fill Value (version 3, late allocation,
    written if set, undefined) and Data Layout (version 3, contiguous)
    messages; the raw data follows the headers.

Array order: ``julia_order=True`` (default) stores an array the way Julia's
HDF5.jl does — the dataspace lists the dimensions in reverse and the bytes
are the array in column-major order — so an (nx, ny, n) Julia-shaped array
reads as (n, ny, nx) in h5py, exactly as the reference's files do.

The reference chunks the event datasets along the event axis (at most 4096
events per chunk); chunking is a storage detail invisible to readers, and
these files store every dataset contiguously.
"""
from __future__ import annotations

import struct
from typing import Dict

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


# ---------------------------------------------------------------------------
# Jenkins lookup3 hashlittle (the checksum of HDF5's version-2 structures)
# ---------------------------------------------------------------------------
def _rot(x: int, k: int) -> int:
    return ((x << k) | (x >> (32 - k))) & 0xFFFFFFFF


def lookup3(data: bytes, initval: int = 0) -> int:
    """Bob Jenkins' lookup3 ``hashlittle`` of ``data`` (public domain, 2006)."""
    M = 0xFFFFFFFF
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & M
    i = 0
    while n > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & M
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & M
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & M
        # mix
        a = (a - c) & M; a ^= _rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= _rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= _rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= _rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= _rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= _rot(b, 4); b = (b + a) & M
        i += 12
        n -= 12
    if n == 0:
        return c
    tail = data[i:i + n] + b"\x00" * (12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M
    b = (b + int.from_bytes(tail[4:8], "little")) & M
    c = (c + int.from_bytes(tail[8:12], "little")) & M
    # final
    c ^= b; c = (c - _rot(b, 14)) & M
    a ^= c; a = (a - _rot(c, 11)) & M
    b ^= a; b = (b - _rot(a, 25)) & M
    c ^= b; c = (c - _rot(b, 16)) & M
    a ^= c; a = (a - _rot(c, 4)) & M
    b ^= a; b = (b - _rot(a, 14)) & M
    c ^= b; c = (c - _rot(b, 24)) & M
    return c


# ---------------------------------------------------------------------------
# Message encodings
# ---------------------------------------------------------------------------
MSG_DATASPACE, MSG_LINK_INFO, MSG_DATATYPE, MSG_FILL, MSG_LINK = 0x01, 0x02, 0x03, 0x05, 0x06
MSG_LAYOUT, MSG_GROUP_INFO, MSG_ATTRIBUTE = 0x08, 0x0A, 0x0C


def _datatype(dt: np.dtype, strlen: int = 0) -> bytes:
    """Datatype message body (version 1)."""
    if strlen:
        # class 3 string: null-terminated (padding type 0), UTF-8 (charset 1)
        return struct.pack("<B3sI", (1 << 4) | 3, bytes([0x10, 0, 0]), strlen)
    dt = np.dtype(dt)
    if dt.kind in "iub":
        signed = 0x08 if dt.kind == "i" else 0
        return struct.pack("<B3sIHH", (1 << 4) | 0, bytes([signed, 0, 0]), dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.itemsize == 4:
            return struct.pack("<B3sIHHBBBBI", (1 << 4) | 1, bytes([0x20, 31, 0]), 4, 0, 32, 23, 8, 0, 23, 127)
        if dt.itemsize == 8:
            return struct.pack("<B3sIHHBBBBI", (1 << 4) | 1, bytes([0x20, 63, 0]), 8, 0, 64, 52, 11, 0, 52, 1023)
    raise TypeError(f"unsupported dtype {dt}")


def _dataspace(dims) -> bytes:
    """Dataspace message body (version 2): scalar for dims == ()."""
    if len(dims) == 0:
        return struct.pack("<BBBB", 2, 0, 0, 0)
    return struct.pack("<BBBB", 2, len(dims), 0, 1) + b"".join(struct.pack("<Q", int(d)) for d in dims)


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    return struct.pack("<BHB", mtype, len(body), flags) + body


def _object_header(messages: bytes, attr_phase: bool = False) -> bytes:
    """Version-2 object header with one chunk: prefix, messages, checksum.
    Flags: chunk-0 size in 4 bytes; optionally attribute phase-change values
    (max compact 64, min dense 6) so that many attributes stay compact."""
    flags = 0x02 | (0x10 if attr_phase else 0)
    pre = b"OHDR" + struct.pack("<BB", 2, flags)
    if attr_phase:
        pre += struct.pack("<HH", 64, 6)
    pre += struct.pack("<I", len(messages))
    body = pre + messages
    return body + struct.pack("<I", lookup3(body))


def _attribute(name: str, value) -> bytes:
    """Attribute message body (version 3)."""
    nm = name.encode("utf-8") + b"\x00"
    if isinstance(value, (str, bytes)):
        s = value.encode("utf-8") if isinstance(value, str) else value
        data = s + b"\x00"
        dtype_b = _datatype(None, strlen=len(data))
        space_b = _dataspace(())
    else:
        a = np.asarray(value)
        if a.dtype == np.bool_:
            a = a.astype(np.uint8)
        dtype_b = _datatype(a.dtype)
        space_b = _dataspace(a.shape[::-1] if a.ndim else ())
        data = np.asfortranarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes(order="F")
    head = struct.pack("<BBHHHB", 3, 0, len(nm), len(dtype_b), len(space_b), 1)
    return head + nm + dtype_b + space_b + data


def write_h5(path: str, datasets: Dict[str, np.ndarray], attrs: Dict[str, object] | None = None,
             julia_order: bool = True) -> None:
    """Write ``datasets`` (name -> array) and root ``attrs`` (name -> str,
    int, float or numpy scalar/array) to a new HDF5 file at ``path``."""
    attrs = attrs or {}
    items = []
    for name, arr in datasets.items():
        a = np.asarray(arr)
        if a.dtype == np.bool_:
            a = a.astype(np.uint8)
        a = a.astype(a.dtype.newbyteorder("<"), copy=False)
        if julia_order:
            dims = a.shape[::-1]
            raw = a.tobytes(order="F")
        else:
            dims = a.shape
            raw = a.tobytes(order="C")
        items.append((name, a.dtype, dims, raw))

    # dataset object headers (their sizes do not depend on addresses)
    def ds_header(dt, dims, addr, size):
        msgs = (_message(MSG_DATASPACE, _dataspace(dims)) +
                _message(MSG_DATATYPE, _datatype(dt), flags=0x01) +
                _message(MSG_FILL, struct.pack("<BB", 3, 0x0A)) +
                _message(MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, addr, size)))
        return _object_header(msgs)

    def root_header(addrs):
        msgs = _message(MSG_LINK_INFO, struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF))
        msgs += _message(MSG_GROUP_INFO, struct.pack("<BBHH", 0, 0x01, 64, 6))
        for (name, *_), addr in zip(items, addrs):
            nb = name.encode("utf-8")
            if len(nb) > 255:
                raise ValueError("dataset names are limited to 255 bytes")
            msgs += _message(MSG_LINK, struct.pack("<BBB", 1, 0x10, 1) + struct.pack("<B", len(nb)) + nb +
                             struct.pack("<Q", addr))
        for k, v in attrs.items():
            msgs += _message(MSG_ATTRIBUTE, _attribute(k, v))
        return _object_header(msgs, attr_phase=True)

    sb_size = 48
    root_size = len(root_header([0] * len(items)))
    pos = sb_size + root_size
    hdr_addrs, hdr_sizes = [], []
    for name, dt, dims, raw in items:
        hdr_addrs.append(pos)
        n = len(ds_header(dt, dims, 0, len(raw)))
        hdr_sizes.append(n)
        pos += n
    data_addrs = []
    for name, dt, dims, raw in items:
        pos = (pos + 7) & ~7
        data_addrs.append(pos)
        pos += len(raw)
    eof = pos
    root = root_header(hdr_addrs)
    assert len(root) == root_size
    sb = SIGNATURE + struct.pack("<BBBBQQQQ", 2, 8, 8, 0, 0, UNDEF, eof, sb_size)
    sb += struct.pack("<I", lookup3(sb))
    with open(path, "wb") as f:
        f.write(sb)
        f.write(root)
        for (name, dt, dims, raw), addr in zip(items, data_addrs):
            f.write(ds_header(dt, dims, addr if len(raw) else UNDEF, len(raw)))
        for (name, dt, dims, raw), addr in zip(items, data_addrs):
            f.write(b"\x00" * (addr - f.tell()))
            f.write(raw)
        assert f.tell() == eof


# ---------------------------------------------------------------------------
# Reader for the subset written above (used by the tests and by users without
# an HDF5 library); verifies every checksum.
# ---------------------------------------------------------------------------
class H5FormatError(ValueError):
    pass


def _parse_datatype(b: bytes):
    cv = b[0]
    cls, ver = cv & 0x0F, cv >> 4
    bits = b[1:4]
    size = struct.unpack_from("<I", b, 4)[0]
    if cls == 0:
        signed = bool(bits[0] & 0x08)
        if bits[0] & 0x01:
            raise H5FormatError("big-endian integers are not supported")
        return np.dtype(("i" if signed else "u") + str(size)).newbyteorder("<"), 8 + 4
    if cls == 1:
        return np.dtype("f" + str(size)).newbyteorder("<"), 8 + 12
    if cls == 3:
        return ("str", size), 8
    raise H5FormatError(f"unsupported datatype class {cls} (version {ver})")


def _parse_dataspace(b: bytes):
    ver, nd, flags, typ = struct.unpack_from("<BBBB", b, 0)
    if ver != 2:
        raise H5FormatError(f"dataspace version {ver}")
    dims = struct.unpack_from("<" + "Q" * nd, b, 4) if nd else ()
    return tuple(int(d) for d in dims)


def _parse_header(buf: bytes, addr: int):
    if buf[addr:addr + 4] != b"OHDR":
        raise H5FormatError(f"no object header at {addr}")
    ver, flags = buf[addr + 4], buf[addr + 5]
    if ver != 2:
        raise H5FormatError("object header version")
    p = addr + 6
    if flags & 0x20:
        p += 16
    if flags & 0x10:
        p += 4
    size_bytes = 1 << (flags & 0x03)
    chunk = int.from_bytes(buf[p:p + size_bytes], "little")
    p += size_bytes
    end = p + chunk
    if end + 4 > len(buf):
        raise H5FormatError(f"object header at {addr} runs past the end of the file")
    stored = struct.unpack_from("<I", buf, end)[0]
    if lookup3(buf[addr:end]) != stored:
        raise H5FormatError(f"object header checksum mismatch at {addr}")
    msgs = []
    while p + 4 <= end:
        mtype, msize, mflags = struct.unpack_from("<BHB", buf, p)
        p += 4
        if flags & 0x04:
            p += 2
        msgs.append((mtype, buf[p:p + msize]))
        p += msize
    return msgs


def _decode(raw: bytes, dt, dims, julia_order: bool):
    if isinstance(dt, tuple):
        s = raw[:dt[1]]
        return s.split(b"\x00", 1)[0].decode("utf-8")
    a = np.frombuffer(raw, dtype=dt)
    if not dims:
        return a[0]
    shape = tuple(dims[::-1]) if julia_order else tuple(dims)
    return a.reshape(shape, order="F" if julia_order else "C")


def read_h5(path: str, julia_order: bool = True):
    """(datasets, attrs) of a file written by ``write_h5``."""
    buf = open(path, "rb").read()
    if buf[:8] != SIGNATURE or buf[8] != 2:
        raise H5FormatError("not a version-2 superblock HDF5 file")
    if lookup3(buf[:44]) != struct.unpack_from("<I", buf, 44)[0]:
        raise H5FormatError("superblock checksum mismatch")
    eof, root_addr = struct.unpack_from("<QQ", buf, 28)
    if eof != len(buf):
        raise H5FormatError("end-of-file address does not match the file size")
    datasets, attrs = {}, {}
    for mtype, body in _parse_header(buf, root_addr):
        if mtype == MSG_LINK:
            ver, fl = body[0], body[1]
            p = 2
            if fl & 0x08:
                p += 1
            if fl & 0x04:
                p += 8
            if fl & 0x10:
                p += 1
            ln_size = 1 << (fl & 0x03)
            ln = int.from_bytes(body[p:p + ln_size], "little")
            p += ln_size
            name = body[p:p + ln].decode("utf-8")
            addr = struct.unpack_from("<Q", body, p + ln)[0]
            dt = dims = layout = None
            for t2, b2 in _parse_header(buf, addr):
                if t2 == MSG_DATATYPE:
                    dt, _ = _parse_datatype(b2)
                elif t2 == MSG_DATASPACE:
                    dims = _parse_dataspace(b2)
                elif t2 == MSG_LAYOUT:
                    ver_l, cls = b2[0], b2[1]
                    if ver_l != 3 or cls != 1:
                        raise H5FormatError("only contiguous layouts are supported")
                    layout = struct.unpack_from("<QQ", b2, 2)
            d_addr, d_size = layout
            raw = buf[d_addr:d_addr + d_size] if d_size else b""
            datasets[name] = _decode(raw, dt, dims, julia_order)
        elif mtype == MSG_ATTRIBUTE:
            ver, fl, nsz, tsz, ssz, cs = struct.unpack_from("<BBHHHB", body, 0)
            p = 9
            name = body[p:p + nsz].split(b"\x00", 1)[0].decode("utf-8")
            p += nsz
            dt, _ = _parse_datatype(body[p:p + tsz])
            p += tsz
            dims = _parse_dataspace(body[p:p + ssz])
            p += ssz
            attrs[name] = _decode(body[p:], dt, dims, julia_order)
    return datasets, attrs
