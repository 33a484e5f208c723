"""Host side of the big-fourier drop-in (big-fourier/src/lib.rs:128-335,
bfpy.pyi): .npy headers written the way big-fourier writes them and the
chunked editor that big-wave's disk vectors use (big-wave/vector.py:115-131)."""

import numpy as np
import pytest

from rave_sim_b200 import bigfourier as bf


@pytest.mark.parametrize("typ,dt", [("c16", np.complex128), ("c8", np.complex64)])
def test_header_is_128_bytes_npy_v1(tmp_path, typ, dt):
    p = tmp_path / "u.npy"
    getattr(bf, f"generate_header_{typ}")(p, 12345)
    raw = p.read_bytes()
    assert len(raw) == 128 and raw[:8] == b"\x93NUMPY\x01\x00" and raw[-1:] == b"\n"
    assert int.from_bytes(raw[8:10], "little") == 118
    # with the data appended numpy reads it back
    x = (np.arange(12345) * (1 + 0.5j)).astype(dt)
    with open(p, "ab") as f:
        f.write(x.tobytes())
    y = np.load(p)
    assert y.dtype == dt and np.array_equal(y, x)


def test_chunked_editor_writes_reads_and_clamps(tmp_path):
    # the write loop of big-wave/vector.py:121-131 over a header-only file
    p = tmp_path / "u.npy"
    n, chunk = 1000, 256
    bf.generate_header_c16(p, n)
    x = (np.arange(n) + 1j * np.arange(n)[::-1]).astype(np.complex128)
    ce = bf.ChunkedEditor(p)
    assert len(ce) == n and ce.position() == 0 and ce.dtype() == "<c16"
    buf = np.empty(chunk, np.complex128)
    written = 0
    while ce.position() < len(ce):
        k = min(chunk, n - ce.position())
        buf[:k] = x[ce.position():ce.position() + k]
        written += ce.write_chunk_c16(buf)
        ce.advance(chunk)
    assert written == n and ce.position() == n
    ce.advance(10)
    assert ce.position() == n
    assert np.array_equal(np.load(p), x)
    ce = bf.ChunkedEditor(p)
    ce.advance(900)
    out = np.zeros(chunk, np.complex128)
    assert ce.read_chunk_c16(out) == 100
    assert np.array_equal(out[:100], x[900:]) and not out[100:].any()
    # the position does not move on read or write
    assert ce.position() == 900


def test_chunked_editor_rejects_wrong_dtype_and_short_files(tmp_path):
    p = tmp_path / "u.npy"
    bf.generate_header_c8(p, 64)
    ce = bf.ChunkedEditor(p)
    with pytest.raises(ValueError):
        ce.write_chunk_c16(np.zeros(8, np.complex128))
    with pytest.raises(ValueError, match="ends earlier"):
        ce.read_chunk_c8(np.zeros(8, np.complex64))
    with pytest.raises(FileNotFoundError):
        bf.ChunkedEditor(tmp_path / "missing.npy")
