"""Out-of-core FFT through the GPU: a drop-in for big-fourier's Python module.

big-wave's disk vectors (big-wave/vector.py:95-146, ``use_disk_vector``) keep
fields larger than memory in .npy files and transform them with big-fourier
(``bfpy``): ``fft_c16`` / ``ifft_c16`` / ``fft_c8`` / ``ifft_c8`` (infile,
outfile, scratchfile), ``generate_header_c16`` / ``_c8`` and
``ChunkedEditor`` (big-fourier/src/lib.rs:65-335, stubs in bfpy.pyi). This
module provides the same functions. The transforms run in the engine
(``rsw_fft_host``): the field is memory-mapped on the host and streams
through a bounded set of device slabs (big-fourier's four-step split,
big-fourier/src/bfft.rs:11-100), so it may exceed the GPU's memory.
``fft_host`` does the same for numpy arrays.

NumPy convention: forward unnormalised, inverse scaled by 1/N.
"""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np

from . import _lib as L
from .engine import _stream_ptr, _torch

HEADER_BYTES = 128
_TYPES = {"c16": np.dtype("<c16"), "c8": np.dtype("<c8")}


def _device_bytes(device_bytes):
    if device_bytes is not None:
        return int(device_bytes)
    torch = _torch()
    free, _ = torch.cuda.mem_get_info()
    return int(min(8 << 30, free * 0.4))


def fft_host(x: np.ndarray, out: np.ndarray | None = None, scratch: np.ndarray | None = None,
             inverse: bool = False, device_bytes: int | None = None) -> np.ndarray:
    """FFT (or inverse FFT) of a 1-D complex128 / complex64 host array of a
    power-of-two length >= 256 through the GPU. ``out`` may be ``x`` when a
    separate ``scratch`` array of the same shape and dtype is given; without
    ``scratch`` the intermediate results go to ``out``. ``device_bytes``
    bounds the device working set (default: 40 % of free memory, at most
    8 GiB)."""
    if x.ndim != 1 or x.dtype not in (np.complex128, np.complex64) or not x.flags.c_contiguous:
        raise ValueError("x must be a contiguous 1-D complex128 or complex64 array")
    if out is None:
        out = np.empty_like(x)
    for a, name in ((out, "out"), (scratch, "scratch")):
        if a is not None and (a.shape != x.shape or a.dtype != x.dtype or not a.flags.c_contiguous
                              or not a.flags.writeable):
            raise ValueError(f"{name} must be a writeable contiguous array like x")
    code = L.RSW_C128 if x.dtype == np.complex128 else L.RSW_C64
    lib = L.load()
    L.check(lib.rsw_fft_host(x.ctypes.data, out.ctypes.data, scratch.ctypes.data if scratch is not None else None,
                             x.size, code, int(bool(inverse)), _device_bytes(device_bytes), _stream_ptr()))
    return out


# ------------------------------------------------------------------ .npy files
def _header(dtype: np.dtype, length: int) -> bytes:
    """NPY version 1.0 header padded to 128 bytes, as big-fourier writes it
    (big-fourier/src/npy/mod.rs:107-124)."""
    fields = "{'descr': '%s', 'fortran_order': False, 'shape': (%d,), }" % (dtype.str, length)
    head = b"\x93NUMPY\x01\x00" + (HEADER_BYTES - 10).to_bytes(2, "little") + fields.encode("latin1")
    if len(head) > HEADER_BYTES - 1:
        raise ValueError("length too large for a 128-byte header")
    return head + b" " * (HEADER_BYTES - 1 - len(head)) + b"\n"


def generate_header_c16(filename: os.PathLike | str, len: int) -> None:  # noqa: A002 (reference name)
    """A .npy file holding only the header of a complex128 vector of ``len``
    entries (truncating the file); the data is appended afterwards."""
    Path(filename).write_bytes(_header(_TYPES["c16"], int(len)))


def generate_header_c8(filename: os.PathLike | str, len: int) -> None:  # noqa: A002 (reference name)
    Path(filename).write_bytes(_header(_TYPES["c8"], int(len)))


def _read_header(path: Path):
    with open(path, "rb") as f:
        version = np.lib.format.read_magic(f)
        read = np.lib.format.read_array_header_1_0 if version == (1, 0) else np.lib.format.read_array_header_2_0
        shape, fortran, dtype = read(f)
        offset = f.tell()
    if len(shape) != 1 or fortran:
        raise ValueError(f"{path}: only one-dimensional arrays are supported")
    return shape[0], np.dtype(dtype), offset


def _transform(infile, outfile, scratchfile, dtype: np.dtype, inverse: bool, device_bytes=None) -> None:
    src, dst, scr = Path(infile), Path(outfile), Path(scratchfile)
    n, dt, off = _read_header(src)
    if dt != dtype:
        raise ValueError(f"{src}: expected dtype {dtype.str}, found {dt.str}")
    if dst.exists() and dst.resolve() == src.resolve():
        # in place: intermediate results in the scratch file, result over the input
        if scr.exists() and scr.resolve() == src.resolve():
            raise ValueError("in-place transforms need a scratch file other than the input")
        x = np.memmap(src, dtype=dt, mode="r+", offset=off, shape=(n,))
        scratch = np.lib.format.open_memmap(scr, mode="w+", dtype=dt, shape=(n,))
        fft_host(x, out=x, scratch=scratch, inverse=inverse, device_bytes=device_bytes)
        x.flush()
        del scratch
        return
    x = np.memmap(src, dtype=dt, mode="r", offset=off, shape=(n,))
    out = np.lib.format.open_memmap(dst, mode="w+", dtype=dt, shape=(n,))
    fft_host(x, out=out, inverse=inverse, device_bytes=device_bytes)
    out.flush()


def fft_c16(infile, outfile, scratchfile, device_bytes=None) -> None:
    _transform(infile, outfile, scratchfile, _TYPES["c16"], False, device_bytes)


def ifft_c16(infile, outfile, scratchfile, device_bytes=None) -> None:
    _transform(infile, outfile, scratchfile, _TYPES["c16"], True, device_bytes)


def fft_c8(infile, outfile, scratchfile, device_bytes=None) -> None:
    _transform(infile, outfile, scratchfile, _TYPES["c8"], False, device_bytes)


def ifft_c8(infile, outfile, scratchfile, device_bytes=None) -> None:
    _transform(infile, outfile, scratchfile, _TYPES["c8"], True, device_bytes)


class ChunkedEditor:
    """Walks over a 1-D complex .npy file in chunks (big-fourier/src/lib.rs:150-335):
    ``read_chunk_*`` / ``write_chunk_*`` transfer up to len(buffer) entries at
    the current position and return the count; ``advance`` moves the position
    (clamped to the length). The file may hold only its header so far
    (``generate_header_*``): writes extend it."""

    def __init__(self, file: os.PathLike | str):
        self._path = Path(file)
        if not self._path.is_file():
            raise FileNotFoundError(str(self._path))
        self._len, self._dtype, self._offset = _read_header(self._path)
        self._pos = 0

    def position(self) -> int:
        return self._pos

    def __len__(self) -> int:
        return self._len

    def advance(self, nr_elements: int) -> None:
        self._pos = min(self._pos + int(nr_elements), self._len)

    def dtype(self) -> str:
        return self._dtype.str

    def _check(self, buffer, typ):
        if self._dtype != _TYPES[typ]:
            raise ValueError(f"file holds {self._dtype.str}, not {_TYPES[typ].str}")
        if buffer.dtype != _TYPES[typ] or buffer.ndim != 1 or not buffer.flags.c_contiguous:
            raise ValueError("the given array is not a contiguous 1-D array of the file's dtype")
        return min(buffer.size, self._len - self._pos)

    def _write(self, buffer, typ) -> int:
        k = self._check(buffer, typ)
        with open(self._path, "r+b") as f:
            f.seek(self._offset + self._pos * self._dtype.itemsize)
            f.write(buffer[:k].tobytes())
        return k

    def _read(self, buffer, typ) -> int:
        k = self._check(buffer, typ)
        with open(self._path, "rb") as f:
            f.seek(self._offset + self._pos * self._dtype.itemsize)
            data = f.read(k * self._dtype.itemsize)
        if len(data) != k * self._dtype.itemsize:
            raise ValueError(f"expected the file to contain {self._len} entries, but it ends earlier")
        buffer[:k] = np.frombuffer(data, dtype=self._dtype)
        return k

    def write_chunk_c16(self, buffer: np.ndarray) -> int:
        return self._write(buffer, "c16")

    def read_chunk_c16(self, buffer: np.ndarray) -> int:
        return self._read(buffer, "c16")

    def write_chunk_c8(self, buffer: np.ndarray) -> int:
        return self._write(buffer, "c8")

    def read_chunk_c8(self, buffer: np.ndarray) -> int:
        return self._read(buffer, "c8")
