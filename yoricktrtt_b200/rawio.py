"""Raw data files of the reference's workflows.

* Simulator float files: a 512-byte header of 128 float32 words followed by
  float32 records (``Tomography_3D/Simul_Data/io.c:24-110`` writes them; the
  reconstruction script reads volume and projections with
  ``raw_read(file, float, nu, nv, 720, offset=512)``,
  ``Tomography_3D/Ytrtt3D_script_reconstructions.i:50-51``).
* Detector frames: signed 16-bit words after a 100-byte header, shifted by
  a constant to the unsigned count (``Tomography_2D/Ytrtt2D_read_real_data.i:10``
  adds 2^15, ``Tomography_2D/Ytrtt2D_batch_real_data.i:31`` adds 2^16 - 1).

Dimensions are given fastest first, as in the reference's ``raw_read`` calls;
the arrays come back in C order, so their shape is the reversed list
(``(nu, nv, n)`` gives ``[n][nv][nu]``).
"""
from __future__ import annotations

import os

import numpy as np

HEADER_BYTES = 512
HEADER_WORDS = HEADER_BYTES // 4

# Named words of the simulator header (io.c:70-97); the others are zero.
HEADER_FIELDS = {
    "min": 0, "max_x1.01": 1, "one": 2, "records": 3, "record_rows": 4,
    "first_data_word": 5,
    "x_pixels": 10, "y_pixels": 11, "z_pixels": 12,
    "x_size": 13, "y_size": 14, "z_size": 15,
    "x_off": 16, "y_off": 17, "z_off": 18,
    "u_pixels": 19, "v_pixels": 20, "u_size": 31, "v_size": 32,
    "u_offsino": 33, "v_offsino": 34, "stretch_factor": 35,
    "dual_points": 43, "dual_radius": 44, "dual_focal": 45,
    "cb_radius": 46, "cb_focal": 47, "cb_points": 48,
}


def read_raw(path, dims, dtype=np.float32, offset=HEADER_BYTES):
    """Array of ``prod(dims)`` elements of ``dtype`` (little-endian) starting
    ``offset`` bytes into the file, shaped ``dims[::-1]``.  The file must
    hold at least that many bytes."""
    dims = [int(d) for d in dims]
    if any(d <= 0 for d in dims):
        raise ValueError(f"dimensions must be positive: {dims}")
    dt = np.dtype(dtype).newbyteorder("<")
    count = int(np.prod(dims))
    need = offset + count * dt.itemsize
    size = os.path.getsize(path)
    if size < need:
        raise ValueError(f"{path}: {size} bytes, {need} needed for {dims} {dt} at offset {offset}")
    a = np.fromfile(path, dtype=dt, count=count, offset=offset)
    return a.reshape(dims[::-1]).astype(dt.newbyteorder("="), copy=False)


def read_header(path):
    """The named words of a simulator file's 512-byte header, as floats."""
    h = np.fromfile(path, dtype="<f4", count=HEADER_WORDS)
    if h.size != HEADER_WORDS:
        raise ValueError(f"{path}: shorter than its {HEADER_BYTES}-byte header")
    return {k: float(h[i]) for k, i in HEADER_FIELDS.items()}


def write_raw(path, data, header=None, record_rows=None):
    """Write ``data`` as float32 after a 512-byte header.  ``header`` (a dict
    of ``HEADER_FIELDS`` names, e.g. from ``read_header``) fills the named
    words; the words the simulator's writer derives from the data are set
    from ``data``: min (at most 0), 1.01 x max, the record count (leading
    dimension), the record height and the first-data-word marker 513."""
    a = np.ascontiguousarray(data, dtype="<f4")
    if a.ndim < 2:
        raise ValueError("data must have at least 2 dimensions (records of rows)")
    words = np.zeros(HEADER_WORDS, dtype="<f4")
    for k, v in (header or {}).items():
        words[HEADER_FIELDS[k]] = v
    words[0] = min(float(a.min()), 0.0)
    words[1] = float(a.max()) * 1.01
    words[2] = 1.0
    words[3] = a.shape[0]
    words[4] = a.shape[1] if record_rows is None else record_rows
    words[5] = HEADER_WORDS * 4 + 1
    with open(path, "wb") as f:
        f.write(words.tobytes())
        f.write(a.tobytes())


def read_detector_frames(paths, nu, nv, offset=100, shift=2.0 ** 15):
    """(len(paths), nv, nu) float64 counts of 16-bit detector frames: each
    file holds nu x nv signed 16-bit words (u fastest) after ``offset``
    header bytes; ``shift`` is added to every word."""
    out = np.empty((len(paths), nv, nu))
    for k, p in enumerate(paths):
        out[k] = read_raw(p, (nu, nv), dtype=np.int16, offset=offset).astype(np.float64) + float(shift)
    return out
