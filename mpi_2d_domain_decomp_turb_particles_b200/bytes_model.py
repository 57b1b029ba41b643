"""Algorithmic bytes of the path's kernels per step: the numerators of the HBM roofline
fractions the benchmark reports.

Droplet update (interpolation + history + drag advance + position update), per droplet:
positions read + written (FP64, 48 B); droplet velocity read + written (24 B mixed /
48 B FP64); velocity history, 2 levels read + 1 written (36 / 72 B); fluid history, 3
levels read + 1 written (48 / 96 B); interpolated velocity written and read (24 / 48 B);
radius or tau_p (4 / 8 B); cell key (4 B).  Total 188 B (mixed) and 324 B (FP64), plus one
pass over the three field components: 3 n^3 * 4 B (mixed, FP32 field) or 3 n^3 * 8 B.
Of these the interpolation kernel moves the field, the positions it reads (24 B) and the
velocity it writes (3 words); the advance kernel the rest.

Flow step (FP64, M = n * n * (n/2 + 1) complex modes): the update kernel reads the
transformed product, N_old and u (3 components each) and writes N_old, u and the six
inputs of the next transforms: 21 complex words = 336 B per mode.  The cross-product
kernel reads u and omega (6 words) and writes u x omega (3 words) per point, 72 B, plus
the droplet context's padded copy of u (3 words of the droplet precision).
"""

PER_DROPLET = {"mixed": 188, "fp64": 324}
FIELD_WORD = {"mixed": 4, "fp64": 8}


def update_bytes(precision: str, n: int, npart: int) -> int:
    return PER_DROPLET[precision] * npart + 3 * n ** 3 * FIELD_WORD[precision]


def interp_bytes(precision: str, n: int, npart: int) -> int:
    w = FIELD_WORD[precision]
    return 3 * n ** 3 * w + (24 + 3 * w) * npart


def advance_bytes(precision: str, n: int, npart: int) -> int:
    return update_bytes(precision, n, npart) - interp_bytes(precision, n, npart)


def flow_update_bytes(n: int) -> int:
    return 336 * n * n * (n // 2 + 1)


def flow_cross_bytes(n: int, emit_precision: str = "mixed") -> int:
    return (72 + 3 * FIELD_WORD[emit_precision]) * n ** 3


def collision_bytes(precision: str, npart: int) -> int:
    """COLLISION_DET reads every owned droplet's packed cell-list entry once (x, y, z,
    radius as FP64 and four ints: 48 B) and its state once (displacement, old and new
    velocity, fluid velocity: 12 words).  A lower bound: the ghost entries (a few per cent
    of the droplets) and the cell start table are not counted."""
    return (48 + 12 * FIELD_WORD[precision]) * npart


# The interpolation's on-chip floor.  Every (droplet, component) evaluates a 6 x 6 x 6
# stencil out of shared memory: 216 loads and 216 FMAs (FP32), or 216 loads, 648 DMUL and
# 216 DADD (FP64, the reference's order ((v * wx) * wy) * wz added term by term).
# Shared memory returns one 128-byte wavefront per SM per clock, one warp-wide FP32 load
# when the lanes fall in distinct banks; the FP64 pipe retires 64 operations per SM per
# clock on B200 (37 TFLOP/s of FP64 FMA over 148 SMs at 1.965 GHz).
STENCIL_POINTS = 216
FP64_OPS_PER_SM_CLOCK = 64


def interp_onchip(precision: str, npart: int, measured_ms: float, num_sms: int, clocks: dict | None) -> dict:
    """Lower bound of the interpolation kernel set by the on-chip unit it leans on (shared
    memory for FP32, the FP64 pipe for FP64) at the SM clock sampled during the run, and
    the fraction of it the measured kernel time reaches."""
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    hz = float(mhz) * 1e6
    tasks = 3 * npart
    if precision == "mixed":
        units = tasks * STENCIL_POINTS / 32.0               # wavefronts at full lane use
        floor_s = units / (num_sms * hz)
        bound = "shared-memory wavefronts (one 32-lane FP32 load per SM per clock)"
        unit_name = "wavefronts"
    else:
        units = tasks * STENCIL_POINTS * 4.0                # 3 DMUL + 1 DADD per term
        floor_s = units / (num_sms * FP64_OPS_PER_SM_CLOCK * hz)
        bound = "FP64 pipe (64 operations per SM per clock)"
        unit_name = "fp64_ops"
    floor_ms = floor_s * 1e3
    return {"bound": bound, unit_name: units, "sm_mhz": float(mhz), "floor_ms": floor_ms,
            "frac": floor_ms / measured_ms if measured_ms and measured_ms > 0 else None}
