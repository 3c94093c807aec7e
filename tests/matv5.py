"""A minimal MAT level-5 file writer for test fixtures, written from the
published MAT-file format (MathWorks, "MAT-File Format", level 5): a 128-byte
header, then one miMATRIX data element per variable.  It shares no code with
uncc_sar_focusing_b200.matdata or scipy's writer, so files written here check
the reader against the format itself: MATLAB's column-major order, nested
structs, single- and double-precision complex arrays, 1 x N and N x 1 vectors.

Values: numpy arrays (2-D after np.atleast_2d; written column-major as MATLAB
stores them), Python floats (1 x 1 double), or dicts (1 x 1 structs).
"""
from __future__ import annotations

import struct

import numpy as np

MI_INT8, MI_UINT8, MI_INT32, MI_UINT32, MI_SINGLE, MI_DOUBLE, MI_MATRIX = 1, 2, 5, 6, 7, 9, 14
MX_STRUCT, MX_DOUBLE, MX_SINGLE = 2, 6, 7
F_COMPLEX = 0x0800


def _element(mi_type: int, payload: bytes) -> bytes:
    pad = (-len(payload)) % 8
    return struct.pack("<II", mi_type, len(payload)) + payload + b"\0" * pad


def _matrix(name: str, value) -> bytes:
    if isinstance(value, dict):
        names = list(value)
        width = 32
        body = _element(MI_UINT32, struct.pack("<II", MX_STRUCT, 0))
        body += _element(MI_INT32, struct.pack("<ii", 1, 1))
        body += _element(MI_INT8, name.encode())
        body += _element(MI_INT32, struct.pack("<i", width))
        body += _element(MI_INT8, b"".join(n.encode().ljust(width, b"\0") for n in names))
        for n in names:
            body += _matrix("", value[n])
        return _element(MI_MATRIX, body)
    a = np.atleast_2d(np.asarray(value))
    single = a.dtype in (np.float32, np.complex64)
    cls, mi = (MX_SINGLE, MI_SINGLE) if single else (MX_DOUBLE, MI_DOUBLE)
    cplx = np.iscomplexobj(a)
    flags = cls | (F_COMPLEX if cplx else 0)
    body = _element(MI_UINT32, struct.pack("<II", flags, 0))
    body += _element(MI_INT32, struct.pack("<" + "i" * a.ndim, *a.shape))
    body += _element(MI_INT8, name.encode())
    real_t = np.float32 if single else np.float64
    col = np.asfortranarray(a)
    body += _element(mi, np.ascontiguousarray(col.real.T, dtype=real_t).tobytes())  # column-major bytes
    if cplx:
        body += _element(mi, np.ascontiguousarray(col.imag.T, dtype=real_t).tobytes())
    return _element(MI_MATRIX, body)


def write(path: str, variables: dict) -> None:
    text = b"MATLAB 5.0 MAT-file, written by tests/matv5.py".ljust(116, b" ")
    header = text + b"\0" * 8 + struct.pack("<H", 0x0100) + b"IM"
    with open(path, "wb") as fh:
        fh.write(header)
        for name, value in variables.items():
            fh.write(_matrix(name, value))
