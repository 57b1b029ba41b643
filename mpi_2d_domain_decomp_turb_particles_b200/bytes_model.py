"""Algorithmic bytes of one droplet update (interpolation + history + drag advance +
position update) per step, the denominator-free numerator of the HBM roofline.

Per droplet: positions read + written (FP64, 48 B); droplet velocity read + written
(24 B mixed / 48 B FP64); velocity history, 2 levels read + 1 written (36 / 72 B); fluid
history, 3 levels read + 1 written (48 / 96 B); interpolated velocity written and read
(24 / 48 B); radius or tau_p (4 / 8 B); cell key (4 B).  Total 188 B (mixed) and 324 B
(FP64).  Plus one pass over the three field components: 3 n^3 * 4 B (mixed, FP32 field)
or 3 n^3 * 8 B (FP64 field).
"""

PER_DROPLET = {"mixed": 188, "fp64": 324}
FIELD_WORD = {"mixed": 4, "fp64": 8}


def update_bytes(precision: str, n: int, npart: int) -> int:
    return PER_DROPLET[precision] * npart + 3 * n ** 3 * FIELD_WORD[precision]
