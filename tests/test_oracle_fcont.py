"""The oracle's continuous-f restatement (oc_props_fcont; no reference
counterpart): theta = 0 is the reference discretisation bit for bit; lnQ is
continuous where N f crosses an integer (the junction step turns from pure A
into pure B smoothly) and smooth inside a step."""
import numpy as np

import oracle as O

M3, D3, N = (8, 12, 10), (2.0, 3.0, 2.5), 20


def _w(seed=0):
    M = int(np.prod(M3))
    rng = np.random.default_rng(seed)
    w = np.zeros(6 * M)
    w[:M] = rng.normal(0, 1.5, M)
    w[M:2 * M] = rng.normal(0, 0.5, M)
    return w


def _lnq(f, ens, cont=True, seed=0):
    d = O.Density(M3, D3, N)
    w = _w(seed)
    q, phis = (d.props_fcont if cont else d.props)(w, N, 0.1, 0.8, f, ens)
    return q, phis, w[2 * w.size // 6:]


def test_theta_zero_is_the_reference_discretisation():
    for ens in (1, 2):
        q0, p0, c0 = _lnq(0.45, ens, cont=False)   # N f = 9 exactly
        q1, p1, c1 = _lnq(0.45, ens, cont=True)
        assert q0 == q1
        np.testing.assert_array_equal(p0, p1)
        np.testing.assert_array_equal(c0, c1)


def test_lnq_continuous_across_a_step_boundary():
    for ens in (1, 2):
        below, _, _ = _lnq(0.5 - 1e-9, ens)   # n1 = 9, theta -> 1: the junction step is pure A
        at, _, _ = _lnq(0.5, ens)             # n1 = 10, theta = 0
        assert abs(below - at) <= 1e-6 * max(1.0, abs(at)), (below, at)


def test_lnq_smooth_inside_a_step():
    f0 = 0.47   # N f = 9.4
    for ens in (1, 2):
        d1 = (_lnq(f0 + 1e-3, ens)[0] - _lnq(f0 - 1e-3, ens)[0]) / 2e-3
        d2 = (_lnq(f0 + 5e-4, ens)[0] - _lnq(f0 - 5e-4, ens)[0]) / 1e-3
        assert abs(d1 - d2) <= 1e-5 * max(1.0, abs(d2)), (d1, d2)
        assert abs(d2) > 1e-6   # f does move lnQ
