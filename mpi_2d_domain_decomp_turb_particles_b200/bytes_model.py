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
