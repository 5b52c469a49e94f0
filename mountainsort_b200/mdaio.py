"""Reader/writer for the MountainSort ``.mda`` array format.

The format (``packages/ms3/mda/mdaio.cpp:60-203``) is a little-endian header

    int32 data_type      -2 uint8, -3 float32, -4 int16, -5 int32, -6 uint16,
                         -7 float64, -8 uint32   (``mda/mdaio.h:55-62``)
    int32 bytes_per_entry
    int32 num_dims       negative => the dims that follow are int64
    dims                 int32 each (or int64 each)

followed by the data in column-major order: element (m, t) of an M x N
timeseries sits at ``m + M*t`` -- the channel index varies fastest
(``pyms/mlpy/mdaio.py:45-46``).  The writer switches to 64-bit dims when any
dimension exceeds 2e9, as ``mda_write_header`` does (``mdaio.cpp:152-156``).

Files are written to ``path + '.tmp'`` and renamed on close, which is how
``DiskWriteMda`` makes outputs atomic (``mda/diskwritemda.cpp:84-85,138-146``).
"""
from __future__ import annotations

import os
import struct

import numpy as np

DT_CODES = {
    -2: np.dtype("uint8"),
    -3: np.dtype("float32"),
    -4: np.dtype("int16"),
    -5: np.dtype("int32"),
    -6: np.dtype("uint16"),
    -7: np.dtype("float64"),
    -8: np.dtype("uint32"),
}
CODE_OF = {v: k for k, v in DT_CODES.items()}
MAX_DIMS = 50


class MdaError(ValueError):
    pass


class MdaHeader:
    __slots__ = ("dt_code", "dtype", "bytes_per_entry", "dims", "header_size", "uses64bitdims")

    def __init__(self, dt_code, dims, uses64bitdims=None):
        if dt_code not in DT_CODES:
            raise MdaError(f"unsupported mda data type code {dt_code}")
        self.dt_code = int(dt_code)
        self.dtype = DT_CODES[dt_code]
        self.bytes_per_entry = self.dtype.itemsize
        self.dims = tuple(int(d) for d in dims)
        if uses64bitdims is None:
            uses64bitdims = any(d > 2e9 for d in self.dims)
        self.uses64bitdims = bool(uses64bitdims)
        self.header_size = 12 + len(self.dims) * (8 if self.uses64bitdims else 4)

    @property
    def size(self) -> int:
        n = 1
        for d in self.dims:
            n *= d
        return n


def read_header(f) -> MdaHeader:
    """Parse an mda header from an open binary file (``mdaio.cpp:60-141``)."""
    raw = f.read(12)
    if len(raw) < 12:
        raise MdaError("truncated mda header")
    dt_code, nbytes, ndims = struct.unpack("<iii", raw)
    if dt_code not in DT_CODES:
        raise MdaError(f"problem with data type: {dt_code}")
    if nbytes <= 0 or nbytes > 8:
        raise MdaError(f"bad bytes per entry: {nbytes}")
    use64 = ndims < 0
    ndims = abs(ndims)
    if ndims == 0 or ndims > MAX_DIMS:
        raise MdaError(f"bad number of dims: {ndims}")
    fmt = "<%dq" % ndims if use64 else "<%di" % ndims
    raw = f.read(struct.calcsize(fmt))
    if len(raw) < struct.calcsize(fmt):
        raise MdaError("truncated mda dims")
    dims = struct.unpack(fmt, raw)
    if any(d < 0 for d in dims):
        raise MdaError(f"negative dimension in {dims}")
    return MdaHeader(dt_code, dims, uses64bitdims=use64)


def write_header(f, hdr: MdaHeader) -> None:
    nd = len(hdr.dims)
    f.write(struct.pack("<iii", hdr.dt_code, hdr.bytes_per_entry, -nd if hdr.uses64bitdims else nd))
    fmt = "<%dq" % nd if hdr.uses64bitdims else "<%di" % nd
    f.write(struct.pack(fmt, *hdr.dims))


def readmda(path: str) -> np.ndarray:
    """Read a whole .mda file into an array with the file's dtype and dims
    (Fortran order, so ``X[m, t]`` is channel m at timepoint t)."""
    with open(path, "rb") as f:
        hdr = read_header(f)
        data = np.fromfile(f, dtype=hdr.dtype, count=hdr.size)
    if data.size != hdr.size:
        raise MdaError(f"short mda file {path}: {data.size} of {hdr.size} entries")
    return data.reshape(hdr.dims, order="F")


def read_header_path(path: str) -> MdaHeader:
    with open(path, "rb") as f:
        return read_header(f)


def writemda(X: np.ndarray, path: str, dtype=None, uses64bitdims=None) -> None:
    """Write ``X`` as .mda (via ``path.tmp`` and an atomic rename).

    Conversion to a narrower integer dtype truncates toward zero like the
    reference's ``std::copy`` (``mdaio.cpp:232-243``)."""
    X = np.asarray(X)
    dt = np.dtype(dtype) if dtype is not None else X.dtype
    if dt not in CODE_OF:
        raise MdaError(f"unsupported dtype {dt}")
    dims = X.shape if X.ndim >= 1 else (1,)
    if len(dims) == 1:
        dims = (dims[0], 1)
    hdr = MdaHeader(CODE_OF[dt], dims, uses64bitdims=uses64bitdims)
    flat = np.reshape(X, -1, order="F")
    if flat.dtype != dt:
        if np.issubdtype(dt, np.integer) and np.issubdtype(flat.dtype, np.floating):
            flat = np.trunc(flat)
        flat = flat.astype(dt)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        write_header(f, hdr)
        flat.tofile(f)
    os.replace(tmp, path)


def timeseries_as_rows(X: np.ndarray) -> np.ndarray:
    """View an M x N Fortran-order timeseries as a C-contiguous N x M array
    (one row of M channels per timepoint), which is the memory layout the
    GPU kernels and the C ABI use.  No copy when X is Fortran-contiguous."""
    return np.asarray(X).T


def timeseries_rows_view(path: str):
    """(M, N, rows) of an M x N .mda timeseries file without reading it:
    rows is a read-only (N, M) memory map of the data in the file's dtype."""
    hdr = read_header_path(path)
    M = hdr.dims[0]
    N = hdr.dims[1] if len(hdr.dims) > 1 else 1
    if M * N == 0:
        return M, N, np.zeros((N, M), dtype=hdr.dtype)
    return M, N, np.memmap(path, dtype=hdr.dtype, mode="r", offset=hdr.header_size, shape=(N, M))


class TimeseriesWriter:
    """An M x N timeseries written block by block into ``path.tmp``, sized in
    full when opened (timepoints never written stay zero, like the
    reference's preallocated file), renamed to ``path`` by close()
    (``mda/diskwritemda.cpp:57-149,255-265``); abort() removes it."""

    def __init__(self, path: str, dtype, M: int, N: int):
        self.path, self.tmp = path, path + ".tmp"
        dt = np.dtype(dtype)
        hdr = MdaHeader(CODE_OF[dt], (M, N))
        with open(self.tmp, "wb") as f:
            write_header(f, hdr)
            f.truncate(hdr.header_size + M * N * dt.itemsize)
        self._rows = (np.memmap(self.tmp, dtype=dt, mode="r+", offset=hdr.header_size, shape=(N, M))
                      if M * N > 0 else None)

    def write(self, t0: int, rows: np.ndarray) -> None:
        self._rows[t0:t0 + len(rows)] = rows

    def close(self) -> None:
        if self._rows is not None:
            self._rows.flush()
            self._rows = None
        os.replace(self.tmp, self.path)

    def abort(self) -> None:
        self._rows = None
        if os.path.exists(self.tmp):
            os.remove(self.tmp)
