"""Accuracy of the shared elementary functions (nexdynipc_b200/csrc/nx_libm.h)
against the C library, in units in the last place.  Both the oracle and the
kernels use them, so their outputs agree bit for bit; this test bounds how far
that common arithmetic is from correctly rounded results."""
import numpy as np

from oracle import refcpu


def ulps(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    sp = np.spacing(np.maximum(np.abs(a), np.abs(b)))
    return np.abs(a - b) / sp


def test_sin_cos():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-np.pi, np.pi, 200000), rng.uniform(-1e-3, 1e-3, 50000),
                        rng.uniform(-50, 50, 50000), [0.0, 1e-300, np.pi / 4, np.pi / 2]])
    assert ulps(refcpu.libm(0, x), np.sin(x)).max() <= 2.0
    assert ulps(refcpu.libm(1, x), np.cos(x)).max() <= 2.0


def test_atan2_first_quadrant_and_signs():
    rng = np.random.default_rng(2)
    y = np.abs(rng.normal(size=200000)) * 10.0 ** rng.uniform(-12, 2, 200000)
    x = np.abs(rng.normal(size=200000)) * 10.0 ** rng.uniform(-12, 2, 200000)
    assert ulps(refcpu.libm(2, y, x), np.arctan2(y, x)).max() <= 2.0
    s = rng.choice([-1.0, 1.0], size=(2, 200000))
    assert ulps(refcpu.libm(2, s[0] * y, s[1] * x), np.arctan2(s[0] * y, s[1] * x)).max() <= 2.0


def test_log_exp_tanh_cosh():
    rng = np.random.default_rng(3)
    x = 10.0 ** rng.uniform(-8, 3, 200000)
    assert ulps(refcpu.libm(3, x), np.log(x)).max() <= 2.0
    t = rng.uniform(-700, 700, 200000)
    assert ulps(refcpu.libm(4, t), np.exp(t)).max() <= 2.0
    s = np.concatenate([rng.uniform(-3, 3, 200000), rng.uniform(-1e-4, 1e-4, 1000)])
    assert ulps(refcpu.libm(5, s), np.tanh(s)).max() <= 3.0
    assert ulps(refcpu.libm(6, s), np.cosh(s)).max() <= 3.0
