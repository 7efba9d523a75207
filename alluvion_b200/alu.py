"""Checkpoint files in the reference's formats, so states move between the
reference and this engine unchanged.

* `.alu` variable files: Variable<D, M>::write_file / read_file
  (variable.hpp:132-262).  Layout: D uint32 shape entries (the outermost
  may be smaller than the variable's when writing a prefix), a uint32 0
  ending the shape, the uint32 number of primitives per element, one type
  label byte ('f' float32, 'd' float64, 'i' int32, 'u' uint32), then the
  elements.  Reading converts float32 files to float64 variables and back,
  as the reference does; any other type mismatch is an error.
* Pile state files: Pile::write_file / read_file (pile.hpp:757-793): per
  body x[3], v[3], q[4] (x, y, z, w), omega[3] of the real type, x, v and
  omega optionally scaled when writing.
"""
import os

import numpy as np

LABELS = {np.dtype(np.float32): b"f", np.dtype(np.float64): b"d",
          np.dtype(np.int32): b"i", np.dtype(np.uint32): b"u"}
TYPES = {v: k for k, v in LABELS.items()}


class AluError(RuntimeError):
    pass


def write_alu(path, array, primitives_per_element=1, shape_outermost=None):
    """Writes `array` ([shape..., primitives] or [shape...] when primitives
    is 1) as an .alu file.  shape_outermost < shape[0] writes a prefix."""
    a = np.ascontiguousarray(array)
    if a.dtype not in LABELS:
        raise AluError("unsupported element type %s" % a.dtype)
    p = int(primitives_per_element)
    shape = list(a.shape[:-1]) if p > 1 else list(a.shape)
    if p > 1 and a.shape[-1] != p:
        raise AluError("last axis %d != primitives per element %d" % (a.shape[-1], p))
    if not shape:
        raise AluError("a variable has at least one dimension")
    outer = shape[0] if shape_outermost is None else int(shape_outermost)
    if outer > shape[0]:
        raise AluError("writing more than the outermost shape (%d > %d)" % (outer, shape[0]))
    with open(path, "wb") as f:
        f.write(np.asarray([outer] + shape[1:] + [0, p], dtype=np.uint32).tobytes())
        f.write(LABELS[a.dtype])
        f.write(a[:outer].tobytes())


def read_alu(path, dims=None, dtype=None):
    """Reads an .alu file.  dims: the variable's number of dimensions D (if
    None, the shape runs to the 0 terminator).  dtype: the variable's
    primitive type; float32 <-> float64 converts.  Returns an array shaped
    [shape..., primitives] (the primitives axis only when > 1)."""
    if not os.path.exists(path):
        raise AluError("Failed to open alu file: %s" % path)
    with open(path, "rb") as f:
        raw = f.read()
    off = 0
    shape = []
    while True:
        if off + 4 > len(raw):
            raise AluError("truncated header: %s" % path)
        v = int(np.frombuffer(raw, np.uint32, 1, off)[0])
        off += 4
        if v == 0:
            break
        shape.append(v)
        if dims is not None and len(shape) > dims:
            raise AluError("dimension mismatch when reading %s" % path)
    if dims is not None and len(shape) != dims:
        raise AluError("shape mismatch when reading %s" % path)
    p = int(np.frombuffer(raw, np.uint32, 1, off)[0])
    off += 4
    label = raw[off:off + 1]
    off += 1
    if label not in TYPES:
        raise AluError("unknown type label %r in %s" % (label, path))
    src = TYPES[label]
    count = int(np.prod(shape)) * p
    if len(raw) - off < count * src.itemsize:
        raise AluError("truncated data: %s" % path)
    data = np.frombuffer(raw, src, count, off).copy()
    if dtype is not None:
        want = np.dtype(dtype)
        if want != src:
            if {want, src} == {np.dtype(np.float32), np.dtype(np.float64)}:
                data = data.astype(want)
            else:
                raise AluError("data type mismatch when reading %s" % path)
    return data.reshape(shape + ([p] if p > 1 else []))


def write_pile(path, rigid, x_scale=1.0, v_scale=1.0, omega_scale=1.0):
    """Pile::write_file: rigid is an (nb, 13) array of x, v, q, omega."""
    r = np.asarray(rigid)
    out = r.copy()
    out[:, 0:3] *= r.dtype.type(x_scale)
    out[:, 3:6] *= r.dtype.type(v_scale)
    out[:, 10:13] *= r.dtype.type(omega_scale)
    with open(path, "wb") as f:
        f.write(np.ascontiguousarray(out).tobytes())


def read_pile(path, dtype=np.float32, num_rigids=None, src_offset=0):
    """Pile::read_file: (nb, 13) array of x, v, q, omega of `dtype`."""
    item = 13 * np.dtype(dtype).itemsize
    with open(path, "rb") as f:
        raw = f.read()
    total = len(raw) // item
    n = total - src_offset if num_rigids is None else min(num_rigids, total - src_offset)
    return np.frombuffer(raw, dtype, 13 * n, src_offset * item).reshape(n, 13).copy()


def pile_size(path, dtype=np.float32):
    """Pile::get_size_from_file."""
    return os.path.getsize(path) // (13 * np.dtype(dtype).itemsize)
