"""The TENO5 smooth-stencil shortcut keeps exactly what the cut-off keeps.

The kernels skip the cut-off when tau = |b0 - b2| <= 4 e_min (e_k = b_k +
eps) and take the linear weights.  These tests replay both cut-off forms in
numpy, on random indicator triples over the whole range the kernels see
(zeros, subnormal-sized, O(1), up to 1e30, mixed scales), and check that
every triple the test passes keeps all three sub-stencils:

* FP32 (teno_keep32x2): x_k = t + s / e_k with t = e_min / (e_min + tau),
  s = tau t, keep iff x_k^6 >= 1e-5 sum x_j^6, eps = FLT_MIN.  The kernel's
  reciprocal is the SFU approximation; here it is the correctly rounded
  one, perturbed by +-2 ulp to cover the approximation's error.
* FP64 (Teno<double>::keep_mask, teno5_pair64): g_k = 1 + tau e_i e_j /
  (e0 e1 e2), keep iff not G_k < 1e-5 sum G, eps = 1e-40.

NaN and infinite indicators must fail the test (they take the cut-off path
and its non-finite flag)."""
import numpy as np

FLT_MIN = np.float32(1.17549435e-38)


def _triples(rng, n, dtype, top):
    scale = 10.0 ** rng.uniform(-40, np.log10(top), (n, 1))
    b = scale * 10.0 ** rng.uniform(-2, 0.7, (n, 3))
    b[rng.random((n, 3)) < 0.05] = 0.0
    same = rng.random(n) < 0.2          # near-equal triples: tau tiny
    b[same] = b[same, :1] * (1 + 1e-3 * rng.standard_normal((same.sum(), 3))) ** 2
    return np.clip(b, 0, top).astype(dtype)


def _smooth32(b):
    with np.errstate(invalid="ignore", over="ignore"):
        em = np.minimum(b[:, 0], np.minimum(b[:, 1], b[:, 2])) + FLT_MIN
        tau = np.abs(b[:, 0] - b[:, 2])
        return (tau <= np.float32(4) * em) & (em <= np.float32(1e30))


def _keep32(b, ulp):
    f = np.float32
    with np.errstate(all="ignore"):
        e = b + FLT_MIN
        tau = np.abs(b[:, 0] - b[:, 2])
        em = e.min(axis=1)

        def rcp(x):
            r = (f(1) / x).astype(f)
            return np.nextafter(r, f(np.inf) if ulp > 0 else f(0)) if ulp else r

        t = em * rcp(em + tau)
        s = tau * t
        x = np.stack([s * rcp(e[:, k]) + t for k in range(3)], axis=1).astype(f)
        y = x * x
        G = (y * y) * y
        lim = f(1e-5) * ((G[:, 0] + G[:, 1]) + G[:, 2])
        return (G >= lim[:, None]).all(axis=1)


def _smooth64(b):
    with np.errstate(invalid="ignore"):
        em = b.min(axis=1) + 1e-40
        tau = np.abs(b[:, 0] - b[:, 2])
        return (tau <= 4.0 * em) & (b.max(axis=1) <= 1e30)


def _keep64(b):
    e = b + 1e-40
    tau = np.abs(b[:, 0] - b[:, 2])
    prod = e[:, 0] * (e[:, 1] * e[:, 2])
    ti = tau / prod
    g = [1.0 + ti * (e[:, 1] * e[:, 2]), 1.0 + ti * (e[:, 0] * e[:, 2]), 1.0 + ti * (e[:, 0] * e[:, 1])]
    G = np.stack([(x * x * x) ** 2 for x in g], axis=1)
    lim = 1e-5 * G.sum(axis=1)
    return (~(G < lim[:, None])).all(axis=1) & np.isfinite(lim)


def test_fp32_smooth_triples_keep_every_substencil():
    rng = np.random.default_rng(11)
    b = _triples(rng, 400_000, np.float32, 1e30)
    ok = _smooth32(b)
    assert ok.sum() > 50_000
    for ulp in (0, 1, -1):
        assert _keep32(b[ok], ulp).all()
    # the threshold is not loose to the point of being meaningless: just past
    # the reach of the test, cut sub-stencils do occur
    assert not _keep32(b[~ok], 0).all()


def test_fp64_smooth_triples_keep_every_substencil():
    rng = np.random.default_rng(12)
    b = _triples(rng, 400_000, np.float64, 1e30)
    ok = _smooth64(b)
    assert ok.sum() > 50_000
    assert _keep64(b[ok]).all()
    assert not _keep64(b[~ok]).all()


def test_non_finite_indicators_fail_the_test():
    bad = np.array([[np.nan, 1, 1], [1, 1, np.nan], [np.inf, 1, 1], [np.inf, np.inf, np.inf],
                    [1, 1, np.inf], [np.inf, 2e38, 3e38]])
    assert not _smooth64(bad).any()
    assert not _smooth32(bad.astype(np.float32)).any()
