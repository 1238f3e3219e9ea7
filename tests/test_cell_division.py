"""The engine's cell-coordinate division (csrc/dpd_kernels.cuh: division_magic,
cell_coords) divides a box-local cell index c < 2^31 by nx and by nx*ny as
floor(c * m / 2^k) with k = 31 + ceil(log2 d), m = ceil(2^k / d).  This test
restates that rule and checks it against integer division for divisors up to
2^31 - 1 and numerators at the edges of every quotient and of the range (the
engine's own cell assignments are compared with the oracle's in every GPU
parity test)."""
import random


def magic(d):
    l = 0
    while (1 << l) < d:
        l += 1
    k = 31 + l
    return ((1 << k) + d - 1) // d, k


def test_division_by_invariant_integers_is_exact():
    rng = random.Random(7)
    divisors = list(range(1, 600)) + [1 << p for p in range(31)] + [(1 << p) - 1 for p in range(2, 32)] + \
        [(1 << p) + 1 for p in range(1, 31)] + [rng.randrange(1, 1 << 31) for _ in range(400)]
    top = (1 << 31) - 1
    for d in divisors:
        m, k = magic(d)
        assert m < (1 << 64) and m * top < (1 << 64)   # the product fits the device's 64-bit multiply
        cs = {0, 1, d - 1, d, d + 1, top, top - 1, top - d}
        q = top // d
        cs.update({q * d, q * d - 1, (q // 2) * d - 1, (q // 2) * d})
        cs.update(rng.randrange(0, top + 1) for _ in range(50))
        for c in cs:
            if 0 <= c <= top:
                assert (c * m) >> k == c // d, (d, c)


def test_cell_coordinates_of_every_cell_of_a_box():
    for nx, ny, nz in [(64, 64, 32), (128, 128, 128), (5, 7, 6), (1, 1, 3), (3, 1, 1)]:
        mx, kx = magic(nx)
        mxy, kxy = magic(nx * ny)
        for cl in range(0, nx * ny * nz, max(1, nx * ny * nz // 20000)):
            q = (cl * mx) >> kx
            iz = (cl * mxy) >> kxy
            assert (cl - q * nx, q - iz * ny, iz) == (cl % nx, (cl // nx) % ny, cl // (nx * ny))
