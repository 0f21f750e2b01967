"""Host-side logic of the batched form (no GPU): the seeded case set and the closed-form
periodic shift the batch kernel derives from its step counter."""
import numpy as np

from periodicshiftlbm_b200.batch import X_EXTENTS, batch_configs

CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1]
CY = [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]
CZ = [0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1]


def test_batch_case_set_follows_the_recipe():
    cfgs = batch_configs(64, seed=2024)
    assert cfgs == batch_configs(64, seed=2024)  # seeded
    assert len({c.nx for c in cfgs}) == 4
    for c in cfgs:
        assert c.nx in X_EXTENTS and c.ny == c.nz == c.nx // 2
        d = 2 * c.radius
        assert d == c.nx / 8
        re = c.u_in * d / c.nu
        assert 1e2 * (1 - 1e-9) <= re <= 1e6 * (1 + 1e-9)
        assert c.smagorinsky == (0.1 if re > 1e3 else 0.0)
        assert c.refine is None


def streamed(shift, d, n):
    """applyStreaming.h:11-31, one step: subtract d, wrap into [0, n) at most twice."""
    s = shift - d
    for _ in range(2):
        if s < 0:
            s += n
    for _ in range(2):
        if s >= n:
            s -= n
    return s


def closed_form(shift0, d, n, step):
    adv = (-d) % n
    return ((step % n) * adv + shift0) % n


def test_closed_form_shift_equals_repeated_streaming():
    rng = np.random.default_rng(5)
    for nx, ny, nz in [(64, 32, 32), (96, 48, 48), (5, 3, 2), (192, 96, 96)]:
        n = nx * ny * nz
        for q in range(27):
            d = CX[q] + nx * CY[q] + nx * ny * CZ[q]
            s = s0 = int(rng.integers(0, n))
            for step in range(1, 400):
                s = streamed(s, d, n)
                assert s == closed_form(s0, d, n, step)
            # far-out step counts (no overflow in 64-bit: (step mod n) * adv < 2^62)
            big = 10 ** 7 + 3
            assert closed_form(s0, d, n, big) == (s0 - big * d) % n
