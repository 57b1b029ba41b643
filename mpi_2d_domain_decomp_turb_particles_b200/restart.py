"""Restart files in the reference's formats (load_save.f90), single rank (rank 0000).

* ``part.NNNN`` (LOAD_PARTICLE / SAVE_PARTICLE, load_save.f90:100-154): record 1 ``nps``
  (INTEGER*4), record 2 ``yp(8,1:nps), fvp(3,0:2,1:nps), fdp(3,0:3,1:nps)`` (REAL*8).
* ``vel2D<idump>.NNNN`` (input_output, load_save.f90:2-51): six records, the spectral
  velocity ``ux, uy, uz`` and the previous nonlinear term ``ox, oy, oz``, each a REAL*8
  array ``(llx, lly, lz) = (n+2, n+2, n)`` in the reference's transposed spectral layout:
  first index kz (FFT order), second index the (re, im) pairs of kx = 0..n/2, third
  index ky (FFT order); entries n+1, n+2 of the first index are zero.
* ``force.<idump>`` (input_outputf, load_save.f90:55-96): ``iseedff``, ``iv(32)``, ``iy``
  (INTEGER*4 records) and ``b1r, b2r, b3r`` (REAL*8 (6,5,5) each, one record).

Fortran unformatted sequential records: a 4-byte signed length before and after each
record.  A record longer than 2**31 - 1 bytes is split into subrecords; the reader follows
the leading markers (a negative one means the record continues in the next subrecord),
and the writer gives every subrecord but the last a negative leading and trailing marker.
"""
from __future__ import annotations

import os
import struct

import numpy as np

_MAXREC = 2 ** 31 - 1


# ------------------------------------------------------------------------------------
# Fortran sequential records
# ------------------------------------------------------------------------------------
def write_records(path, records, max_record=_MAXREC):
    """records: iterable of numpy arrays or bytes, written in order."""
    with open(path, "wb") as f:
        for r in records:
            data = r.tobytes(order="C") if isinstance(r, np.ndarray) else bytes(r)
            if len(data) == 0:
                f.write(struct.pack("<i", 0) * 2)
                continue
            pos = 0
            while pos < len(data):
                chunk = data[pos:pos + max_record]
                pos += len(chunk)
                more = pos < len(data)
                marker = -len(chunk) if more else len(chunk)
                f.write(struct.pack("<i", marker))
                f.write(chunk)
                f.write(struct.pack("<i", marker))


def read_records(path):
    """All records of the file as bytes objects (subrecords joined)."""
    out = []
    with open(path, "rb") as f:
        buf = f.read()
    pos = 0
    while pos < len(buf):
        parts = []
        while True:
            (m,) = struct.unpack_from("<i", buf, pos)
            n = abs(m)
            parts.append(buf[pos + 4:pos + 4 + n])
            pos += 8 + n
            if m >= 0:
                break
        out.append(b"".join(parts))
    return out


# ------------------------------------------------------------------------------------
# file names (load_save.f90:14-31, 72-78, 112-120)
# ------------------------------------------------------------------------------------
def particle_file(destination, rank=0):
    return os.path.join(destination, f"part.{rank:04d}")


def flow_file(directvelo, idump, rank=0):
    if not 0 <= idump < 100:
        raise ValueError("idump must be 0..99")
    return os.path.join(directvelo, f"vel2D{idump}.{rank:04d}")


def forcing_file(directfor, idump):
    if not 0 <= idump < 100:
        raise ValueError("idump must be 0..99")
    return os.path.join(directfor, f"force.{idump}")


# ------------------------------------------------------------------------------------
# particles
# ------------------------------------------------------------------------------------
def write_particles(path, yp, fvp, fdp):
    nps = yp.shape[0]
    body = np.concatenate([np.ascontiguousarray(yp, np.float64).ravel(), np.ascontiguousarray(fvp, np.float64).ravel(),
                           np.ascontiguousarray(fdp, np.float64).ravel()])
    write_records(path, [np.array([nps], np.int32), body])


def read_particles(path):
    """(yp (nps, 8), fvp (nps, 3, 3), fdp (nps, 4, 3)) in the reference's memory order."""
    r = read_records(path)
    nps = int(np.frombuffer(r[0], np.int32)[0])
    body = np.frombuffer(r[1], np.float64)
    if body.size != nps * (8 + 9 + 12):
        raise ValueError(f"{path}: record 2 holds {body.size} values, expected {nps * 29}")
    yp = body[:nps * 8].reshape(nps, 8).copy()
    fvp = body[nps * 8:nps * 17].reshape(nps, 3, 3).copy()
    fdp = body[nps * 17:].reshape(nps, 4, 3).copy()
    return yp, fvp, fdp


def save_particles(path, partlib):
    s = partlib.get_particles()
    write_particles(path, s["yp"], s["fvp"], s["fdp"])


def load_particles(path, partlib):
    yp, fvp, fdp = read_particles(path)
    partlib.set_particles(yp, fvp, fdp)


# ------------------------------------------------------------------------------------
# spectral velocity: reference layout <-> (3, n, n, n/2+1) complex (kz, ky, kx)
# ------------------------------------------------------------------------------------
def spectral_to_reference(uh):
    """(n, n, n/2+1) complex [kz, ky, kx] -> C array (lz, lly, llx) = Fortran v(llx, lly, lz)."""
    n = uh.shape[0]
    R = np.zeros((n, n + 2, n + 2))
    t = np.transpose(uh, (1, 2, 0))          # [ky, kx, kz]
    R[:, 0::2, :n] = t.real
    R[:, 1::2, :n] = t.imag
    return R


def reference_to_spectral(R):
    n = R.shape[0]
    t = R[:, 0::2, :n] + 1j * R[:, 1::2, :n]   # [ky, kx, kz]
    return np.ascontiguousarray(np.transpose(t, (2, 0, 1)))


def write_flow(path, uh, nold):
    write_records(path, [spectral_to_reference(uh[c]) for c in range(3)] +
                  [spectral_to_reference(nold[c]) for c in range(3)])


def read_flow(path, n):
    r = read_records(path)
    if len(r) != 6:
        raise ValueError(f"{path}: {len(r)} records, expected 6")
    arrs = [np.frombuffer(x, np.float64).reshape(n, n + 2, n + 2) for x in r]
    uh = np.stack([reference_to_spectral(a) for a in arrs[:3]])
    nold = np.stack([reference_to_spectral(a) for a in arrs[3:]])
    return uh, nold


def save_flow(path, flow):
    uh, nold = flow.spectral()
    write_flow(path, uh, nold)


def load_flow(path, flow):
    uh, nold = read_flow(path, flow.n)
    flow.set_spectral(uh, nold)


# ------------------------------------------------------------------------------------
# stochastic forcing state
# ------------------------------------------------------------------------------------
def write_forcing(path, b, iseedf, iyf, ivf):
    """b: (3, 5, 5, 6) = b1r, b2r, b3r, each Fortran (6,5,5)."""
    write_records(path, [np.array([iseedf], np.int32), np.asarray(ivf, np.int32).reshape(32),
                         np.array([iyf], np.int32), np.ascontiguousarray(b, np.float64).ravel()])


def read_forcing(path):
    r = read_records(path)
    iseedf = int(np.frombuffer(r[0], np.int32)[0])
    ivf = np.frombuffer(r[1], np.int32).copy()
    iyf = int(np.frombuffer(r[2], np.int32)[0])
    b = np.frombuffer(r[3], np.float64).reshape(3, 5, 5, 6).copy()
    return b, iseedf, iyf, ivf


def save_forcing(path, flow):
    b, seed, iy, iv = flow.forcing_state()
    write_forcing(path, b, seed, iy, iv)


def load_forcing(path, flow):
    import ctypes as C
    b, seed, iy, iv = read_forcing(path)
    b = np.ascontiguousarray(b, np.float64)
    iv = np.ascontiguousarray(iv, np.int32)
    flow._chk(flow.lib.dl_flow_set_forcing_state(flow.h, b.ctypes.data_as(C.POINTER(C.c_double)), seed, iy,
                                                 iv.ctypes.data_as(C.POINTER(C.c_int))))
