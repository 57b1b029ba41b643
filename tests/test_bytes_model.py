"""The algorithmic byte counts behind the roofline fractions the benchmark reports."""
from mpi_2d_domain_decomp_turb_particles_b200 import bytes_model as bm


def test_update_bytes_split_into_interpolation_and_advance():
    for prec, word, per in (("mixed", 4, 188), ("fp64", 8, 324)):
        n, npart = 256, 1_000_000
        assert bm.update_bytes(prec, n, npart) == per * npart + 3 * n ** 3 * word
        assert bm.interp_bytes(prec, n, npart) + bm.advance_bytes(prec, n, npart) == bm.update_bytes(prec, n, npart)
        # the interpolation moves the field, the positions it reads and the velocity it writes
        assert bm.interp_bytes(prec, n, npart) == 3 * n ** 3 * word + (24 + 3 * word) * npart
    # headline figures quoted in the bench line
    assert bm.update_bytes("mixed", 256, 1_000_000) == 389_326_592
    assert bm.update_bytes("fp64", 256, 1_000_000) == 726_653_184


def test_flow_and_collision_bytes():
    assert bm.flow_update_bytes(256) == 336 * 256 * 256 * 129
    assert bm.flow_cross_bytes(512) == 84 * 512 ** 3
    assert bm.collision_bytes("mixed", 1_000_000) == 96_000_000
    assert bm.collision_bytes("fp64", 10) == 10 * (48 + 96)
