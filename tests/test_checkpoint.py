"""Checkpoint files on the host, without a device (mbt_checkpoint_check):
a well-formed file is accepted and reports its turn; truncated, corrupted,
foreign and overlong files are refused before any device would be touched.
The files are built here in the layout mbt_checkpoint_save writes (header,
records of id + size + bytes, 64-bit FNV-1a checksum of all that precedes
it); exact resume on the device is tests/test_gpu_checkpoint.py."""
import struct

import pytest

from mbtrack_b200 import api

FNV_OFFSET, FNV_PRIME = 1469598103934665603, 1099511628211


def fnv1a(data):
    h = FNV_OFFSET
    for b in data:
        h ^= b
        h = (h * FNV_PRIME) & 0xFFFFFFFFFFFFFFFF
    return h


def build(turn=1234, nbunch=3, records=None, magic=b"MBTCKPT1", version=2):
    """A checkpoint in the writer's layout: the ring-state record (id 17)
    starts with the turn count."""
    if records is None:
        records = [(0, bytes(48)), (17, struct.pack("<q", turn) + bytes(40))]
    key = struct.pack("<14i", nbunch, 64, 3, 16, 0, 8, 2, 1, 1, 0, 64, 0, 0, 0) + struct.pack("<QQ", 7, 9)
    body = magic + struct.pack("<II", version, len(records)) + key
    for rid, data in records:
        body += struct.pack("<IQ", rid, len(data)) + data
    return body + struct.pack("<Q", fnv1a(body))


def test_well_formed_file_is_accepted(tmp_path, libmbt):
    p = tmp_path / "ok.ckpt"
    p.write_bytes(build(turn=1234, nbunch=3))
    assert api.checkpoint_check(str(p)) == (1234, 3)


@pytest.mark.parametrize("damage", ["truncated", "bitflip", "magic", "version", "overlong_record", "trailing",
                                    "empty"])
def test_damaged_files_are_refused(tmp_path, libmbt, damage):
    good = build()
    if damage == "truncated":
        data = good[:-20]
    elif damage == "bitflip":
        b = bytearray(good)
        b[100] ^= 0x10
        data = bytes(b)
    elif damage == "magic":
        data = build(magic=b"MBTCKPT0")
    elif damage == "version":
        data = build(version=1)     # the previous format
    elif damage == "overlong_record":
        # a record claiming more bytes than the file holds (checksum valid)
        body = good[:-8]
        hdr = 8 + 8 + 72
        rid, n = struct.unpack_from("<IQ", body, hdr)
        body = body[:hdr] + struct.pack("<IQ", rid, 1 << 40) + body[hdr + 12:]
        data = body + struct.pack("<Q", fnv1a(body))
    elif damage == "trailing":
        body = good[:-8] + b"xxxx"
        data = body + struct.pack("<Q", fnv1a(body))
    else:
        data = b""
    p = tmp_path / ("bad_%s.ckpt" % damage)
    p.write_bytes(data)
    with pytest.raises(api.MbtError) as e:
        api.checkpoint_check(str(p))
    assert e.value.code == -8   # MBT_ERR_IO


def test_missing_file(tmp_path, libmbt):
    with pytest.raises(api.MbtError):
        api.checkpoint_check(str(tmp_path / "nothing.ckpt"))
