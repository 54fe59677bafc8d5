"""Snapshot files in the reference's formats (oracle).

Restates mod_fft.f90:
  2249-2301  MSAVEX     (one Fortran unformatted sequential file)
  2303-2388  MPISAVEX   (FN.info header records + FN raw COMPLEX(P8), one process)
  2416-2501  MLOADX     2503-2633  MPILOADX
Little-endian, 4-byte record markers, INTEGER 4 bytes, REAL(P8) 8 bytes, the
layout tests/postproc/read_binary_info.ipynb reads.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""

import struct

import numpy as np


def _rec(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def _read(f):
    (n,) = struct.unpack("<i", f.read(4))
    data = f.read(n)
    (m,) = struct.unpack("<i", f.read(4))
    if m != n or len(data) != n:
        raise ValueError("bad Fortran record")
    return data


def msave(path, g, A, glb=True):
    """MSAVEX (glb) or MPISAVEX (not glb) of field A (E in the reference layout)."""
    E = np.asfortranarray(A.E)
    hdr = open(path if glb else path + ".info", "wb")
    with hdr as f:
        if glb:
            _rec(f, struct.pack("<iii", g.NR, g.NTH, g.NX))
            _rec(f, struct.pack("<iii", g.NRCHOP, g.NTCHOP, g.NXCHOP))
        else:
            _rec(f, struct.pack("<iii", g.NDIMR, g.NDIMTH, g.NDIMX))
            _rec(f, struct.pack("<iii", g.NRCHOPDIM, g.NTCHOPDIM, g.NXCHOPDIM))
        _rec(f, struct.pack("<id", A.space, A.LN))
        _rec(f, struct.pack("<dd", g.ZLEN, g.ELL))
        _rec(f, struct.pack("<ii", 1, 0))
        if glb:
            _rec(f, struct.pack("<iii", *E.shape))
            _rec(f, E.tobytes(order="F"))
    if not glb:
        with open(path, "wb") as f:
            f.write(E.tobytes(order="F"))


def mload(path, glb=True, shape=None):
    """MLOADX / MPILOADX: returns (E, space, LN, header dict); the MPI form
    needs the array shape of its space (the .info holds the dims, not the shape)."""
    hdr = {}
    with open(path if glb else path + ".info", "rb") as f:
        a = struct.unpack("<iii", _read(f))
        b = struct.unpack("<iii", _read(f))
        space, ln = struct.unpack("<id", _read(f))
        hdr["zlen"], hdr["ell"] = struct.unpack("<dd", _read(f))
        hdr["minc"], hdr["mklink"] = struct.unpack("<ii", _read(f))
        hdr["dims"], hdr["chops"] = a, b
        if glb:
            shape = struct.unpack("<iii", _read(f))
            E = np.frombuffer(_read(f), dtype=np.complex128).reshape(shape, order="F")
    if not glb:
        E = np.fromfile(path, dtype=np.complex128).reshape(shape, order="F")
    return E, space, ln, hdr
