"""Pins the oracle's integral engine (oracle/ints.c) without Simint: Boys
values against mpmath, closed forms, normalisation, permutation symmetry and
angular-momentum raising checked by finite differences of lower integrals."""
import ctypes

import mpmath
import numpy as np
import pytest

import oracle

L = oracle.lib()


class Shell(ctypes.Structure):
    _fields_ = [("am", ctypes.c_int), ("nprim", ctypes.c_int), ("x", ctypes.c_double), ("y", ctypes.c_double),
                ("z", ctypes.c_double), ("alpha", ctypes.c_void_p), ("coef", ctypes.c_void_p)]


_keep = []


def shell(am, xyz, alphas, coefs, normalize=True):
    a = np.array(alphas, dtype=np.float64)
    c = np.array(coefs, dtype=np.float64)
    if normalize:
        cn = np.zeros_like(c)
        L.oi_normalize(am, len(a), a.ctypes.data, c.ctypes.data, cn.ctypes.data)
        c = cn
    _keep.extend([a, c])
    return Shell(am, len(a), xyz[0], xyz[1], xyz[2], a.ctypes.data, c.ctypes.data)


def nc(l):
    return (l + 1) * (l + 2) // 2


def eri(A, B, C, D):
    out = np.zeros(nc(A.am) * nc(B.am) * nc(C.am) * nc(D.am))
    L.oi_eri(ctypes.byref(A), ctypes.byref(B), ctypes.byref(C), ctypes.byref(D), out.ctypes.data_as(ctypes.c_void_p))
    return out.reshape(nc(A.am), nc(B.am), nc(C.am), nc(D.am))


def ovl(A, B):
    out = np.zeros(nc(A.am) * nc(B.am))
    L.oi_overlap(ctypes.byref(A), ctypes.byref(B), out.ctypes.data_as(ctypes.c_void_p))
    return out.reshape(nc(A.am), nc(B.am))


@pytest.mark.parametrize("m", [0, 1, 3, 6, 8])
@pytest.mark.parametrize("T", [0.0, 1e-9, 0.3, 2.5, 11.7, 29.9, 45.0, 99.9, 100.1, 250.0])
def test_boys_vs_mpmath(m, T):
    F = oracle.boys(8, T)[m]
    if T == 0.0:
        ref = mpmath.mpf(1) / (2 * m + 1)
    else:
        ref = mpmath.quad(lambda t: t ** (2 * m) * mpmath.exp(-T * t * t), [0, 1])
    assert abs(F - float(ref)) <= 1e-14 * max(1.0, abs(float(ref)))


def test_ssss_same_centre_closed_form():
    # four normalised s Gaussians, exponent 1, one centre: 2/sqrt(pi)
    s = shell(0, (0.1, -0.2, 0.3), [1.0], [1.0])
    assert abs(eri(s, s, s, s)[0, 0, 0, 0] - 2.0 / np.sqrt(np.pi)) < 1e-14


def test_ss_overlap_two_centres_closed_form():
    a, b, R = 0.8, 1.3, 1.7
    A = shell(0, (0, 0, 0), [a], [1.0])
    B = shell(0, (0, 0, R), [b], [1.0])
    ref = (2 * np.sqrt(a * b) / (a + b)) ** 1.5 * np.exp(-a * b / (a + b) * R * R)
    assert abs(ovl(A, B)[0, 0] - ref) < 1e-15


@pytest.mark.parametrize("l", [0, 1, 2, 3])
def test_axis_component_normalised(l):
    # contracted shell: the x^l component has unit norm
    A = shell(l, (0.3, 0.1, -0.4), [3.1, 0.9, 0.25], [0.2, 0.5, 0.6])
    S = ovl(A, A)
    assert abs(S[0, 0] - 1.0) < 1e-13
    assert np.allclose(S, S.T, atol=1e-15)


def test_eri_permutation_symmetry():
    A = shell(2, (0.0, 0.1, 0.2), [1.1, 0.3], [0.4, 0.7])
    B = shell(1, (1.0, -0.5, 0.3), [0.9], [1.0])
    C = shell(2, (-0.7, 0.2, 1.1), [0.6], [1.0])
    D = shell(0, (0.2, 0.9, -0.8), [1.7, 0.4], [0.5, 0.6])
    abcd = eri(A, B, C, D)
    assert np.allclose(abcd, eri(B, A, C, D).transpose(1, 0, 2, 3), atol=1e-14)
    assert np.allclose(abcd, eri(A, B, D, C).transpose(0, 1, 3, 2), atol=1e-14)
    assert np.allclose(abcd, eri(C, D, A, B).transpose(2, 3, 0, 1), atol=1e-14)


def test_eri_translation_invariance():
    sh = [(2, (0.0, 0.1, 0.2), [1.1]), (1, (1.0, -0.5, 0.3), [0.9]), (3, (-0.7, 0.2, 1.1), [0.6]), (0, (0, 0, 0), [0.0])]
    d = np.array([0.37, -1.2, 2.5])
    X = [shell(l, c, a, [1.0], normalize=(a[0] > 0)) for l, c, a in sh]
    Y = [shell(l, tuple(np.array(c) + d), a, [1.0], normalize=(a[0] > 0)) for l, c, a in sh[:3]] + [X[3]]
    # the unit shell (exponent 0) has no centre dependence
    assert np.allclose(eri(*X), eri(*Y), atol=1e-13)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_angular_raising_by_finite_difference(axis):
    # d/dA_i of an unnormalised s primitive = 2a * (p_i primitive): check (p s|s s)
    a = 0.9
    A0 = np.array([0.2, -0.1, 0.4])
    B = shell(0, (1.0, 0.5, -0.3), [0.7], [1.0], normalize=False)
    C = shell(1, (-0.6, 0.8, 0.1), [1.3], [1.0], normalize=False)
    D = shell(0, (0.3, 0.3, 0.9), [0.5], [1.0], normalize=False)
    h = 1e-5
    vals = []
    for sgn in (1, -1):
        Ah = A0.copy()
        Ah[axis] += sgn * h
        vals.append(eri(shell(0, tuple(Ah), [a], [1.0], normalize=False), B, C, D)[0, 0])
    fd = (vals[0] - vals[1]) / (2 * h)
    # p primitive with coefficient 1 is unnormalised (x - Ax) e^{-a r^2}; p_x, p_y, p_z = components 0, 1, 2
    P = shell(1, tuple(A0), [a], [1.0], normalize=False)
    p = eri(P, B, C, D)[axis, 0]
    assert np.allclose(fd, 2 * a * p, rtol=1e-7, atol=1e-11)
