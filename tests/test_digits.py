"""The sort kernels' signed-digit recoding (read_bits and signed_digit in
snarkrs_b200/csrc/msm.cu), restated line for line on Python integers: for every
window width the sorts accept (c in [4, 24], W = ceil(255 / c) windows), every
digit lies in [-2^(c-1), 2^(c-1)], so |d| - 1 indexes one of 2^(c-1) buckets,
and sum_w d_w 2^(c w) gives the scalar back for every scalar below the BN254
scalar modulus, the top window included (255 recoding bits leave it no borrow).
The GPU parity tests check the CUDA code itself."""
import random

import oracle as O


def read_bits(words, off, width):
    idx = off >> 5
    if idx >= 8:
        return 0
    sh = off & 31
    w = words[idx]
    if idx + 1 < 8:
        w |= words[idx + 1] << 32
    return (w >> sh) & ((1 << width) - 1)


def signed_digit(words, w, c):
    off = w * c
    b = read_bits(words, off, c)
    d = b - ((b >> (c - 1)) << c)
    carry = read_bits(words, off - 1, 1) if off else 0
    return d + carry


def test_signed_digits_reconstruct_every_scalar():
    rng = random.Random(12)
    scalars = [0, 1, 2, O.R_MOD - 1, O.R_MOD - 2, (1 << 253) - 1, 1 << 253, (1 << 254) - 1]
    scalars += [rng.randrange(O.R_MOD) for _ in range(300)]
    scalars += [(1 << rng.randrange(254)) - 1 for _ in range(50)]   # runs of ones carry through every window
    for c in range(4, 25):
        W = (255 + c - 1) // c   # msm_windows
        for s in scalars:
            words = [(s >> (32 * i)) & 0xFFFFFFFF for i in range(8)]
            digits = [signed_digit(words, w, c) for w in range(W)]
            assert all(-(1 << (c - 1)) <= d <= (1 << (c - 1)) for d in digits), (c, s)
            assert all(d == 0 or 0 <= abs(d) - 1 < (1 << (c - 1)) for d in digits)
            assert sum(d << (c * w) for w, d in enumerate(digits)) == s, (c, s)
