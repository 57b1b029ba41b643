"""Reference restart formats (load_save.f90): Fortran sequential records with subrecords,
the part.NNNN record layout, the transposed spectral layout of vel2D files and the
stochastic forcing record.  CPU only."""
import struct

import numpy as np

from mpi_2d_domain_decomp_turb_particles_b200 import restart


def test_records_round_trip_with_subrecords(tmp_path):
    p = tmp_path / "r.bin"
    recs = [np.arange(5, dtype=np.int32), np.linspace(0, 1, 100), b"", np.array([7], np.int32)]
    restart.write_records(p, recs, max_record=64)
    out = restart.read_records(p)
    assert out[0] == recs[0].tobytes() and out[1] == recs[1].tobytes() and out[2] == b"" and out[3] == recs[3].tobytes()
    raw = open(p, "rb").read()
    assert struct.unpack_from("<i", raw, 0)[0] == 20 and struct.unpack_from("<i", raw, 24)[0] == 20
    # the 800-byte record is split: first subrecord marker negative
    assert struct.unpack_from("<i", raw, 28)[0] == -64


def test_particle_file_layout(tmp_path):
    rng = np.random.default_rng(0)
    yp, fvp, fdp = rng.random((7, 8)), rng.random((7, 3, 3)), rng.random((7, 4, 3))
    p = tmp_path / "part.0000"
    restart.write_particles(p, yp, fvp, fdp)
    raw = open(p, "rb").read()
    # record 1: nps as INTEGER*4; record 2: yp(8,1:nps) then fvp then fdp
    assert struct.unpack_from("<iii", raw, 0) == (4, 7, 4)
    assert struct.unpack_from("<i", raw, 12)[0] == 7 * 29 * 8
    assert struct.unpack_from("<d", raw, 16)[0] == yp[0, 0] and struct.unpack_from("<d", raw, 24)[0] == yp[0, 1]
    y2, v2, d2 = restart.read_particles(p)
    assert np.array_equal(y2, yp) and np.array_equal(v2, fvp) and np.array_equal(d2, fdp)


def test_spectral_layout_known_mode_and_round_trip(tmp_path):
    n = 8
    x = np.arange(n) * 2 * np.pi / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.cos(X) + 0.25 * np.sin(2 * Y) + 0.5 * np.cos(Z)
    uh = np.fft.rfftn(u) / n ** 3                 # [kz, ky, kx], forward normalised 1/n^3
    R = restart.spectral_to_reference(uh)          # Fortran v(llx, lly, lz) as C (lz, lly, llx)
    # cos(x): kx = 1 -> pair index 2 (real part), ky = 0, kz = 0
    assert abs(R[0, 2, 0] - 0.5) < 1e-15
    # cos(z): kz = 1 -> first index 1, kx = 0 real part, ky = 0
    assert abs(R[0, 0, 1] - 0.25) < 1e-15
    # sin(2y): ky = 2 -> third index 2, kx = 0 imag part (-i/2 * 0.25)
    assert abs(R[2, 1, 0] - (-0.125)) < 1e-15
    assert not R[:, :, n:].any()
    assert np.array_equal(restart.reference_to_spectral(R), uh)
    p = tmp_path / "vel2D1.0000"
    restart.write_flow(p, np.stack([uh, 2 * uh, 3 * uh]), np.stack([uh, uh, uh]))
    a, b = restart.read_flow(p, n)
    assert np.array_equal(a[2], 3 * uh) and np.array_equal(b[0], uh)
    assert restart.flow_file("/d/", 1) == "/d/vel2D1.0000" and restart.particle_file("/d/") == "/d/part.0000"


def test_forcing_record(tmp_path):
    b = np.random.default_rng(1).random((3, 5, 5, 6))
    p = tmp_path / "force.3"
    restart.write_forcing(p, b, -232300, 17, np.arange(32))
    b2, seed, iy, iv = restart.read_forcing(p)
    assert np.array_equal(b2, b) and seed == -232300 and iy == 17 and np.array_equal(iv, np.arange(32))
    recs = restart.read_records(p)
    assert [len(r) for r in recs] == [4, 128, 4, 450 * 8]
