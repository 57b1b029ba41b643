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


def test_interp_onchip_floor():
    clk = {"sm_mhz": 1965.0}
    m = bm.interp_onchip("mixed", 1_000_000, 0.2, 148, clk)
    # 3 tasks per droplet x 216 loads / 32 lanes per wavefront, one wavefront per SM per clock
    assert m["wavefronts"] == 3 * 216 * 1_000_000 / 32
    assert abs(m["floor_ms"] - m["wavefronts"] / (148 * 1965e6) * 1e3) < 1e-12
    assert abs(m["frac"] - m["floor_ms"] / 0.2) < 1e-12
    f = bm.interp_onchip("fp64", 1_000_000, 0.5, 148, clk)
    assert f["fp64_ops"] == 3 * 216 * 4 * 1_000_000
    assert abs(f["floor_ms"] - f["fp64_ops"] / (148 * 64 * 1965e6) * 1e3) < 1e-12
    # without a clock record the nominal maximum clock is used
    assert bm.interp_onchip("mixed", 10, 1.0, 148, None)["sm_mhz"] == 1965.0
