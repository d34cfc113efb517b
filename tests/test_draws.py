"""The draws header's own sine/cosine and the reference's random walk
(include/ppc_draws.h), evaluated by the oracle library on the host: accuracy
against libm, and the walk's construction step by step (reference:
src/solver/host/solver_helper.h:82-86,160-165,250-267, src/cell.cpp:128-161).
The device evaluates the same header; the GPU parity tests of division and
motility check it bit for bit against these host values."""
import math

import numpy as np

from oracle import oracle as orc


def _ulp_err(got, want):
    """Error in units of the last place of the correctly rounded value (libm's
    result stands in for it; glibc's sin and cos are within an ulp)."""
    scale = np.spacing(np.maximum(np.abs(want), 2.0 ** -1022))
    return np.abs(got - want) / scale


def test_sincos_against_libm():
    rng = np.random.default_rng(1)
    theta = np.concatenate([
        rng.random(200000) * 2 * np.pi,                                   # the walks' range
        np.array([0.0, np.pi / 4, np.pi / 2, np.pi, 3 * np.pi / 2, 2 * np.pi - 1e-16, 1e-300, 5e-8]),
        np.arange(1, 9) * (np.pi / 4),                                      # octant edges
        rng.uniform(-2 ** 19, 2 ** 19, 20000),                              # the whole domain
    ])
    sn, cs = orc.sincos(theta)
    ws = np.array([math.sin(x) for x in theta])
    wc = np.array([math.cos(x) for x in theta])
    # near a zero of sin or cos the value is tiny and its ulp tinier still:
    # there the error is measured against the argument's rounding (|theta| ulp)
    abs_tol = np.spacing(np.abs(theta)) * 2
    es = np.minimum(_ulp_err(sn, ws), np.abs(sn - ws) / np.maximum(abs_tol, 1e-300))
    ec = np.minimum(_ulp_err(cs, wc), np.abs(cs - wc) / np.maximum(abs_tol, 1e-300))
    assert es.max() <= 2.0, es.max()
    assert ec.max() <= 2.0, ec.max()
    # most values agree with libm exactly
    main = slice(0, 200000)
    assert np.mean(sn[main] == ws[main]) > 0.8
    assert np.mean(cs[main] == wc[main]) > 0.8
    assert np.all(sn[main] ** 2 + cs[main] ** 2 - 1 < 4e-16)


def test_random_walk_construction():
    """ppc_random_walk follows position_helper<dims>::random_walk with the
    counter-based draws in place of the generator: 1-D a sign, 2-D
    (cos, sin) of theta = u * 2 pi, 3-D theta as in 2-D and z = u' * 2 - 1 with
    (cos theta sqrt(1 - z^2), sin theta sqrt(1 - z^2), z)."""
    seed, epoch, rep = 12345, 7, 0
    for slot in range(300):
        u0 = orc.uniform(seed, epoch, rep, slot, 16)
        u1 = orc.uniform(seed, epoch, rep, slot, 17)
        w1 = orc.random_walk(1, seed, epoch, rep, slot, 16)
        assert w1[0] == (-1.0 if u0 < 0.5 else 1.0)
        theta = u0 * (2 * math.pi - 0.0) + 0.0
        sn, cs = orc.sincos(np.array([theta]))
        w2 = orc.random_walk(2, seed, epoch, rep, slot, 16)
        assert w2[0] == cs[0] and w2[1] == sn[0]
        z = u1 * (1.0 - (-1.0)) + (-1.0)
        r = math.sqrt(1 - z * z)
        w3 = orc.random_walk(3, seed, epoch, rep, slot, 16)
        assert w3[0] == cs[0] * r and w3[1] == sn[0] * r and w3[2] == z
        np.testing.assert_allclose(w2, (math.cos(theta), math.sin(theta)), rtol=0, atol=3e-16)


def test_uniform_sphere_and_circle():
    seed = 99
    w3 = np.array([orc.random_walk(3, seed, 0, 0, i, 16) for i in range(20000)])
    np.testing.assert_allclose(np.linalg.norm(w3, axis=1), 1.0, rtol=0, atol=4e-16)
    assert np.all(np.abs(w3.mean(axis=0)) < 0.03)
    # z uniform on [-1, 1] (Archimedes): the variance of z is 1/3
    assert abs(np.var(w3[:, 2]) - 1 / 3) < 0.02
    w2 = np.array([orc.random_walk(2, seed, 0, 0, i, 16) for i in range(20000)])
    np.testing.assert_allclose(np.linalg.norm(w2, axis=1), 1.0, rtol=0, atol=4e-16)
    assert np.all(np.abs(w2.mean(axis=0)) < 0.03)
