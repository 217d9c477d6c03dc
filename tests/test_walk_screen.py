"""The walk decides most candidates with an FP32 screen and only the rest with
the exact FP64 predicate (gizmo_b200/csrc/grid.cu, `screen`). Its margin is
scr = 8 x 2^-24 x box: positions lie in [0, box), so rounding a position to
FP32 and each FP32 subtraction are within 2^-24 box, and an FP32 separation
is within 6 x 2^-24 box of the FP64 one over three axes.

This test restates the screen in numpy float32 arithmetic (IEEE round to
nearest, as the kernel's separate operations; a fused multiply-add there is
only more accurate) and checks, on random pairs placed within a few ulp of the
search radius and across the periodic faces, that every FP32 decision agrees
with the FP64 predicate the CPU search applies.
"""
import numpy as np
import pytest


def _sep2_fp64(xi, xj, box):
    d = xi - xj
    d = np.where(d > 0.5 * box, d - box, np.where(d < -0.5 * box, d + box, d))
    return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]


def _screen_fp32(xi, xj, R, box, positive):
    f = np.float32
    boxf, halff = f(box), f(0.5) * f(box)
    scr = f(4.77e-7) * boxf
    d = xi.astype(f) - xj.astype(f)
    d = np.where(d > halff, d - boxf, np.where(d < -halff, d + boxf, d)).astype(f)
    r2f = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]).astype(f)
    # R rounded up to FP32 (the kernel's __double2float_ru)
    Rf = R.astype(f)
    Rf = np.where(Rf.astype(np.float64) < R, np.nextafter(Rf, f(np.inf)), Rf).astype(f)
    hi = (Rf + scr).astype(f)
    lo = (Rf - scr).astype(f)
    out = np.full(len(R), 2)
    out[r2f > hi * hi] = 0
    inside = (lo > 0) & (r2f < lo * lo)
    if positive:
        inside &= r2f > f(4) * scr * scr
    out[(out == 2) & inside] = 1
    return out


@pytest.mark.parametrize("box", [1.0, 3.7, 1e-3, 1e3])
@pytest.mark.parametrize("positive", [False, True])
def test_fp32_screen_never_contradicts_fp64(box, positive):
    rng = np.random.default_rng(11)
    n = 400_000
    xi = rng.uniform(0, box, (n, 3))
    xi[: n // 4, 0] = rng.uniform(0, 1e-6, n // 4) * box  # near a lower face
    xi[n // 4: n // 2, 1] = box - rng.uniform(0, 1e-6, n // 4) * box  # near an upper face
    R = rng.uniform(1e-5, 5e-2, n) * box
    u = rng.standard_normal((n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    # separations within a few ulp of the radius, on both sides
    r = R * (1.0 + rng.uniform(-3e-7, 3e-7, n))
    xj = (xi + u * r[:, None]) % box
    xj = np.minimum(xj, np.nextafter(box, 0.0))
    r2 = _sep2_fp64(xi, xj, box)
    exact = (r2 < R * R) & ((r2 > 0) if positive else True)
    sc = _screen_fp32(xi, xj, R, box, positive)
    assert not np.any(exact & (sc == 0)), "screen rejected an FP64 neighbour"
    assert not np.any(~exact & (sc == 1)), "screen accepted an FP64 non-neighbour"
    assert (sc == 2).mean() > 0.5  # the samples sit in the band: most are left to FP64
    # and far from the radius the screen decides by itself
    r_far = R * np.where(rng.uniform(size=n) < 0.5, 0.9, 1.1)
    xj2 = np.minimum((xi + u * r_far[:, None]) % box, np.nextafter(box, 0.0))
    sc2 = _screen_fp32(xi, xj2, R, box, positive)
    r2b = _sep2_fp64(xi, xj2, box)
    exact2 = (r2b < R * R) & ((r2b > 0) if positive else True)
    assert (sc2 != 2).mean() > 0.99
    assert np.array_equal(sc2[sc2 != 2] == 1, exact2[sc2 != 2])
