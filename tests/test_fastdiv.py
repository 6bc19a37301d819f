"""The FFT kernels replace runtime integer division by a multiply-high (fft_smem.cuh: make_fastdiv/fdiv):
m = ceil(2^(31+l)/d), l = ceil(log2 d), q = umulhi(n, m) >> (l-1).  This checks the identity, in exact integer
arithmetic, over every divisor and dividend range the kernels use (d <= 4096, n < 2^22)."""
import random


def fastdiv(n, d):
    if d <= 1:
        return n
    l = (d - 1).bit_length()
    m = ((1 << (31 + l)) + d - 1) // d
    assert m < (1 << 32)
    return ((n * m) >> 32) >> (l - 1)


def test_fastdiv_identity():
    rng = random.Random(7)
    for d in range(1, 4097):
        for n in list(range(0, 4096)) + [rng.randrange(0, 1 << 22) for _ in range(64)] + [(1 << 22) - 1]:
            assert fastdiv(n, d) == n // d, (n, d)
