"""PHOENIX matrix files: read the text, NumPy (.npy), PHOENIX binary (.ash) and
MATLAB v4 (.mat) files that the command line writes (and that the reference's
FileHandler::outputMatrixToFile writes, source/system/filehandler.cpp:233-313),
and write them byte for byte as the command line does, through libphx_io.so.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
_io = None


def _lib():
    global _io
    if _io is None:
        path = os.path.join(_PKG, "libphx_io.so")
        if not os.path.exists(path):
            raise OSError(f"{path} is missing: build it with `python -m phoenix_b200.build`")
        lib = C.CDLL(path)
        lib.phxio_encode.restype = C.c_longlong
        lib.phxio_encode.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_uint32, C.c_uint32,
                                     C.POINTER(C.c_uint32), C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_void_p)]
        lib.phxio_free.argtypes = [C.c_void_p]
        lib.phxio_envelope.restype = C.c_int
        lib.phxio_envelope.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                       C.c_void_p, C.c_char_p, C.c_int]
        _io = lib
    return _io


_HEADER = re.compile(r"#\s*SIZE\s+(\d+)\s+(\d+)\s*(.*?)\s*::")


def read_txt(path, complex_=None):
    """A text matrix: (array of shape (N_r, N_c), header dict).  A file with 2 N_r
    value rows is complex (real block, then imaginary block) unless complex_ says."""
    with open(path) as f:
        first = f.readline()
        m = _HEADER.match(first)
        if not m:
            raise ValueError(f"{path}: not a PHOENIX text matrix")
        n_c, n_r = int(m.group(1)), int(m.group(2))
        toks = m.group(3).split()
        k = toks.index("OSC") if "OSC" in toks else len(toks)
        header = {}
        for part in (toks[:k], toks[k + 1:]):
            header.update({part[i]: float(part[i + 1]) for i in range(0, len(part) - 1, 2)})
        rows = [np.array(line.split(), dtype=np.float64) for line in f if line.strip() and not line.startswith("#")]
    data = np.array(rows)
    if complex_ is None:
        complex_ = data.shape[0] == 2 * n_r
    if complex_:
        return data[:n_r] + 1j * data[n_r:2 * n_r], header
    return data[:n_r], header


def _read_binary(path, magic):
    with open(path, "rb") as f:
        raw = f.read()
    if raw[0] != 0x93 or raw[1:1 + len(magic)] != magic:
        raise ValueError(f"{path}: not a {magic.decode()} file")
    off = 1 + len(magic) + 2
    hlen = raw[off] | (raw[off + 1] << 8)
    header = raw[off + 2:off + 2 + hlen].decode("latin1")
    descr = re.search(r"'descr': '([<>|]?)(\w+)'", header).group(2)
    shape = tuple(int(x) for x in re.search(r"'shape': \(([^)]*)\)", header).group(1).split(",") if x.strip())
    dt = {"c8": np.complex64, "c16": np.complex128, "f4": np.float32, "f8": np.float64}[descr]
    data = np.frombuffer(raw[off + 2 + hlen:], dtype=dt)
    return data[:int(np.prod(shape))].reshape(shape)


def read_npy(path):
    return _read_binary(path, b"NUMPY")


def read_ash(path):
    return _read_binary(path, b"PHOENIX")


def read_mat(path):
    """MATLAB v4 as the command line writes it: the element size is taken from
    the file length (its type field says double for single-precision runs too)."""
    with open(path, "rb") as f:
        raw = f.read()
    typ, rows, cols, imagf, namelen = np.frombuffer(raw[128:148], dtype=np.int32)
    body = raw[148 + namelen:]
    n = int(rows) * int(cols) * (2 if imagf else 1)
    dt = np.float32 if len(body) == 4 * n else np.float64
    v = np.frombuffer(body, dtype=dt)
    re_ = v[:rows * cols].reshape(cols, rows).T
    if imagf:
        return re_ + 1j * v[rows * cols:2 * rows * cols].reshape(cols, rows).T
    return re_.copy()


def read_matrix(path):
    """Any of the four formats, by extension: the array (N_r, N_c)."""
    ext = os.path.splitext(path)[1]
    if ext == ".txt":
        return read_txt(path)[0]
    if ext == ".npy":
        return read_npy(path)
    if ext == ".ash":
        return read_ash(path)
    if ext == ".mat":
        return read_mat(path)
    raise ValueError(f"{path}: unknown matrix format")


def encode_matrix(fmt, array, header=(0, 0, 0, 0, 0, 0, 0, 0), precision=-1, window=None, increment=1):
    """The bytes the command line writes for `array` (N_r, N_c) in format fmt
    ("txt", "npy", "ash", "mat"); the array's dtype (complex64/128, float32/64)
    is the run's precision.  header = (L_x, L_y, dx, dy, t, t0, freq, sigma);
    window = (c0, c1, r0, r1)."""
    a = np.ascontiguousarray(array)
    cplx = np.iscomplexobj(a)
    dtype = 0 if a.dtype in (np.float32, np.complex64) else 1
    n_r, n_c = a.shape
    c0, c1, r0, r1 = window if window is not None else (0, n_c, 0, n_r)
    win = (C.c_uint32 * 5)(c0, c1, r0, r1, increment)
    hd = (C.c_double * 8)(*[float(x) for x in header])
    out = C.c_void_p()
    n = _lib().phxio_encode(fmt.encode(), dtype, int(cplx), a.ctypes.data, n_c, n_r, win, hd, int(precision), C.byref(out))
    if n < 0:
        raise RuntimeError("phxio_encode failed")
    try:
        return C.string_at(out, n)
    finally:
        _lib().phxio_free(out)


def evaluate_envelope(args, family, dtype="f64", group=-1, pol="plus", default=0.0):
    """One envelope family of a command line (list of arguments as the
    executable takes them, with --N and --L) on its grid: complex (N_r, N_c)."""
    argv = (C.c_char_p * len(args))(*[a.encode() for a in args])
    n_c, n_r = 400, 400
    if "--N" in args:
        k = args.index("--N")
        n_c, n_r = int(float(args[k + 1])), int(float(args[k + 2]))
    cdt = np.complex64 if dtype == "f32" else np.complex128
    out = np.zeros((n_r, n_c), dtype=cdt)
    err = C.create_string_buffer(512)
    p = {"plus": 1, "minus": 2, "both": 3}[pol]
    st = _lib().phxio_envelope(len(args), argv, family.encode(), 0 if dtype == "f32" else 1, group, p, default,
                               out.ctypes.data, err, 512)
    if st < 0:
        raise ValueError(err.value.decode())
    return out
