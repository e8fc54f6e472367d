"""SLC measurement TIFF ingest (slc_reader.rs): the oracle against the
reference's own reader tests (slc_reader.rs:619-731, restated on synthetic
files since the S1A fixtures are not here), and the GPU reader against the
oracle byte for byte, into host and device memory."""
import struct

import numpy as np
import pytest

import oracle
import sardine_b200 as sd
from sardine_b200 import _abi

SHORT, LONG = 3, 4


def write_slc_tiff(path, iq, le=True, so_type=LONG, magic=42, tags=None, gap_at=None):
    """A Sentinel-1-style measurement TIFF: one IFD, one row per strip,
    contiguous CInt16 rows.  `tags` overrides/adds (tag -> (type, value));
    gap_at inserts 4 bytes before that row (non-contiguous strips)."""
    h, w = iq.shape[:2]
    e = "<" if le else ">"
    entries = {256: (LONG, w), 257: (LONG, h), 258: (SHORT, 32), 259: (SHORT, 1), 277: (SHORT, 1),
               278: (LONG, 1), 339: (SHORT, 5)}
    entries.update(tags or {})
    n = len(entries) + 1
    ifd_at = 8
    table_at = ifd_at + 2 + 12 * n + 4
    each = 2 if so_type == SHORT else 4
    data_at = table_at + (each * h if h > 1 else 0)
    offs = [data_at + r * w * 4 + (4 if gap_at is not None and r >= gap_at else 0) for r in range(h)]
    out = bytearray((b"II" if le else b"MM") + struct.pack(e + "HI", magic, ifd_at))
    out += struct.pack(e + "H", n)
    for tag in sorted(list(entries) + [273]):
        if tag == 273:
            val = offs[0] if h == 1 else table_at
            out += struct.pack(e + "HHI", 273, so_type, h) + (struct.pack(e + "I", val) if so_type == LONG or h > 1
                                                               else struct.pack(e + "HH", val, 0))
        else:
            typ, val = entries[tag]
            out += struct.pack(e + "HHI", tag, typ, 1)
            out += struct.pack(e + "HH", val, 0) if typ == SHORT else struct.pack(e + "I", val)
    out += struct.pack(e + "I", 0)
    assert len(out) == table_at
    if h > 1:
        out += b"".join(struct.pack(e + ("H" if each == 2 else "I"), o) for o in offs)
    for r in range(h):
        if gap_at is not None and r == gap_at:
            out += b"\0" * 4
        out += iq[r].astype(e + "i2").tobytes()
    with open(path, "wb") as f:
        f.write(bytes(out))


def make_minimal_tiff(entries):
    """slc_reader.rs:663-700: header, one IFD of inline entries, one data byte."""
    out = bytearray(b"II" + struct.pack("<HI", 42, 8) + struct.pack("<H", len(entries)))
    for tag, typ, count, val in sorted(entries):
        out += struct.pack("<HHI", tag, typ, count)
        out += struct.pack("<HH", val, 0) if typ == SHORT else struct.pack("<I", val)
    out += struct.pack("<I", 0) + b"\0"
    return bytes(out)


def _iq(h, w, seed):
    rng = np.random.default_rng(seed)
    return np.clip(np.round(rng.normal(0, 60, (h, w, 2))), -32768, 32767).astype(np.int16)


# ── oracle vs the reference's reader tests ──────────────────────────────────
def test_oracle_open_errors(tmp_path):
    assert oracle.slc_read("/nonexistent/path/file.tiff", read=False)[0] == _abi.SD_ERR_SLC_IO   # 629-633
    p = tmp_path / "empty.tiff"
    p.write_bytes(b"")
    assert oracle.slc_read(str(p), read=False)[0] in (_abi.SD_ERR_SLC_IO, _abi.SD_ERR_SLC_NOT_TIFF)  # 635-644
    p.write_bytes(b"This is not a TIFF file at all!!!")
    assert oracle.slc_read(str(p), read=False)[0] == _abi.SD_ERR_SLC_NOT_TIFF  # 646-660
    p.write_bytes(make_minimal_tiff([(256, LONG, 1, 10), (257, LONG, 1, 1), (258, SHORT, 1, 32),
                                     (259, SHORT, 1, 1), (273, LONG, 1, 9999), (277, SHORT, 1, 2),
                                     (278, LONG, 1, 1), (339, SHORT, 1, 5)]))
    assert oracle.slc_read(str(p), read=False)[0] == _abi.SD_ERR_SLC_UNSUPPORTED_FORMAT  # 702-731


CASES = {  # file variant -> the error SlcReader::open gives, or 0
    "plain": ({}, 0),
    "big_endian": ({"le": False}, 0),
    "short_offsets": ({"so_type": SHORT}, 0),
    "bigtiff": ({"magic": 43}, _abi.SD_ERR_SLC_BIGTIFF),
    "compressed": ({"tags": {259: (SHORT, 5)}}, _abi.SD_ERR_SLC_UNSUPPORTED_FORMAT),
    "float32": ({"tags": {339: (SHORT, 3)}}, _abi.SD_ERR_SLC_UNSUPPORTED_FORMAT),
    "rows_per_strip": ({"tags": {278: (LONG, 2)}}, _abi.SD_ERR_SLC_UNSUPPORTED_FORMAT),
    "no_sample_format": ({"tags": {339: (5, 0)}}, _abi.SD_ERR_SLC_MISSING_TAG),
    "gap": ({"gap_at": 7}, _abi.SD_ERR_SLC_NON_CONTIGUOUS_STRIPS),
}


def _make(tmp_path, name, h=180, w=37):
    kw, rc = CASES[name]
    iq = _iq(h, w, len(name))
    if kw.get("so_type") == SHORT:
        h, w = 40, 9  # SHORT offsets must stay below 65536
        iq = _iq(h, w, 1)
    p = str(tmp_path / f"{name}.tiff")
    write_slc_tiff(p, iq, **kw)
    return p, iq, rc


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reader_cases(tmp_path, name):
    p, iq, rc = _make(tmp_path, name)
    got = oracle.slc_read(p, read=False)
    assert got[0] == rc
    if rc:
        return
    h, w = iq.shape[:2]
    assert got[1:3] == (w, h)
    # bursts of 20 lines (the reference's 9 x 1498-line layout, scaled down), the last one exactly at the end
    for first in range(0, h, 20):
        rc2, _, _, rows = oracle.slc_read(p, first, min(20, h - first))
        assert rc2 == 0 and np.array_equal(rows, iq[first:first + 20])
    assert oracle.slc_read(p, h, 1)[0] == _abi.SD_ERR_SLC_LINE_OUT_OF_BOUNDS      # one line past the end
    assert oracle.slc_read(p, h - 2, 10)[0] == _abi.SD_ERR_SLC_LINE_OUT_OF_BOUNDS  # overflow
    assert oracle.slc_read(p, 0, 1)[3].shape == (1, w, 2)                           # one row


# ── GPU reader vs the oracle ────────────────────────────────────────────────
@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_reader_matches_oracle(ctx, tmp_path, name):
    import torch
    p, iq, rc = _make(tmp_path, name)
    if rc:
        with pytest.raises(sd.SlcReadError) as e:
            sd.SlcReader.open(p, ctx=ctx)
        assert e.value.code == rc
        return
    with sd.SlcReader.open(p, ctx=ctx) as r:
        h, w = iq.shape[:2]
        assert (r.width, r.height) == (w, h)
        for first in (0, 20, h - 20):
            host = r.read_burst_raw(first, 20)
            assert np.array_equal(host, oracle.slc_read(p, first, 20)[3])
            dev = torch.empty((20, w, 2), dtype=torch.int16, device="cuda")
            r.read_burst_raw(first, 20, out=dev)
            assert np.array_equal(dev.cpu().numpy(), host)
        assert np.array_equal(r.read_burst_complex(3, 2), iq[3:5].astype(np.float32))
        for first, n in ((h, 1), (h - 2, 10)):
            with pytest.raises(sd.SlcReadError) as e:
                r.read_burst_raw(first, n)
            assert e.value.kind == "LineOutOfBounds"


@pytest.mark.gpu
@pytest.mark.parametrize("le", [True, False])
def test_gpu_reader_streams_large_reads(ctx, tmp_path, le):
    """More than one 32 MB pinned chunk: every chunk lands where it belongs."""
    import torch
    h, w = 3001, 3000  # 36 MB
    iq = _iq(h, w, 9)
    p = str(tmp_path / "large.tiff")
    write_slc_tiff(p, iq, le=le)
    with sd.SlcReader.open(p, ctx=ctx) as r:
        assert r.little_endian == le
        dev = torch.empty((h, w, 2), dtype=torch.int16, device="cuda")
        r.read_burst_raw(0, h, out=dev)
        assert torch.equal(dev.cpu(), torch.from_numpy(iq))
        dev2 = torch.empty((h - 1001, w, 2), dtype=torch.int16, device="cuda")
        r.read_burst_raw(1001, h - 1001, out=dev2)
        assert torch.equal(dev2.cpu(), torch.from_numpy(iq[1001:]))
