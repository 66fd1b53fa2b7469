"""Known-answer checks of the oracle: closed forms and an independent numpy
restatement of density::props (density.h:344-459)."""
import numpy as np
import pytest

import oracle as O


def np_props(wm, wp, m, D, Ns, alpha, phic, f, ens):
    """Independent numpy restatement of props with numpy.fft."""
    M = int(np.prod(m))
    n1 = int(np.floor(Ns * f + 0.5))
    n2, Nh, ds = Ns - n1, int(alpha * Ns), 1.0 / Ns
    k = [np.fft.fftfreq(m[0], 1 / m[0]), np.fft.fftfreq(m[1], 1 / m[1]), np.arange(m[2] // 2 + 1)]
    K0, K1, K2 = np.meshgrid(*k, indexing="ij")
    k2 = 4 * np.pi ** 2 * (K0 ** 2 / D[0] ** 2 + K1 ** 2 / D[1] ** 2 + K2 ** 2 / D[2] ** 2)
    G2, G1 = np.exp(-k2 * ds / 12), np.exp(-k2 * ds / 6)
    wA, wB = wm + wp, wp - wm

    def step(q, w):
        E4 = np.exp(-w * ds / 4)
        E2 = E4 * E4
        a = np.fft.irfftn(np.fft.rfftn(q * E4) * G2, s=m, axes=(0, 1, 2)) * E2
        a = np.fft.irfftn(np.fft.rfftn(a) * G2, s=m, axes=(0, 1, 2))
        b = np.fft.irfftn(np.fft.rfftn(q * E2) * G1, s=m, axes=(0, 1, 2))
        return (4 * a * E4 - b * E2) / 3

    q, qd = [np.ones(m)], [np.ones(m)]
    for s in range(Ns):
        q.append(step(q[-1], wA if s < n1 else wB))
        qd.append(step(qd[-1], wB if s < n2 else wA))
    Q2, QC = qd[Nh].mean(), q[Ns].mean()
    if ens == 1:
        lnQ = phic * np.log(QC) + (1 - phic) / alpha * np.log(Q2)
        zB, zC = (1 - phic) / (Q2 * alpha), phic / QC
    else:
        zB, zC = 1.0, phic
        lnQ = zB * Q2 + zC * QC
    rhB, rCA, rCB = 2 * qd[Nh], qd[Ns] + q[n1] * qd[n2], q[Ns] + q[n1] * qd[n2]
    for lo, hi, acc in ((1, Nh, "h"), (1, n1, "A"), (n1 + 1, Ns, "B")):
        wt = 4
        for s in range(lo, hi):
            if acc == "h":
                rhB = rhB + wt * qd[s] * qd[Nh - s]
            elif acc == "A":
                rCA = rCA + wt * q[s] * qd[Ns - s]
            else:
                rCB = rCB + wt * q[s] * qd[Ns - s]
            wt = 6 - wt
    rhB, rCA, rCB = rhB * zB * ds / 3, rCA * zC * ds / 3, rCB * zC * ds / 3
    return lnQ, np.stack([rCA, rhB + rCB, rhB, rCB]).reshape(4, M)


@pytest.mark.parametrize("m,D,Ns,f,ens,amp", [
    ((8, 8, 8), (4, 4, 4), 20, 0.5, 1, 1.0),
    ((12, 10, 6), (3, 2.5, 2), 21, 0.45, 2, 2.0),
    ((6, 5, 9), (2, 2, 3), 17, 0.3, 1, 3.0),
])
def test_props_matches_numpy_restatement(m, D, Ns, f, ens, amp):
    rng = np.random.default_rng(Ns)
    M = int(np.prod(m))
    wm, wp = rng.normal(0, amp, m), rng.normal(0, amp, m)
    lnQ, conc = np_props(wm, wp, m, D, Ns, 0.2, 0.8, f, ens)
    d = O.Density(m, D, Ns)
    w = np.zeros(6 * M)
    w[:M], w[M:2 * M] = wm.ravel(), wp.ravel()
    lnQ2, phis = d.props(w, Ns, 0.2, 0.8, f, ens)
    assert abs(lnQ - lnQ2) <= 1e-12 * max(1, abs(lnQ))
    assert np.abs(conc - w[2 * M:].reshape(4, M)).max() <= 1e-12


def test_uniform_field_closed_form():
    """W- = a, W+ = b: every Richardson step multiplies q by exp(-w ds) exactly."""
    m, D, Ns, f, alpha, phic = (4, 6, 8), (2, 3, 4), 20, 0.4, 0.1, 0.7
    a, b = 0.7, -0.3
    M = int(np.prod(m))
    d = O.Density(m, D, Ns)
    w = np.zeros(6 * M)
    w[:M], w[M:2 * M] = a, b
    lnQ, phis = d.props(w, Ns, alpha, phic, f, 1)
    n1, ds = 8, 1.0 / Ns
    wA, wB = a + b, b - a
    QC = np.exp(-(wA * n1 + wB * (Ns - n1)) * ds)
    Q2 = np.exp(-wB * int(alpha * Ns) * ds)
    assert abs(lnQ - (phic * np.log(QC) + (1 - phic) / alpha * np.log(Q2))) < 1e-13
    qNs = d.q(0, Ns)
    assert np.allclose(qNs, QC, rtol=1e-13)
    # composite Simpson of a constant integrand with even counts is exact:
    # total copolymer density equals phic, homopolymer (1-phic) * Nh/(alpha N)
    assert abs(phis[0] - phic) < 1e-12
    assert abs(phis[4] - (1 - phic)) < 1e-12


def test_reduction_sum_order():
    rng = np.random.default_rng(0)
    a = rng.normal(size=5000)
    assert abs(O.reduction_sum(a) - a.sum()) < 1e-11


def test_spline_reproduces_linear_data_and_derivative():
    x = np.array([0.0, 0.1, 0.35, 0.6, 1.0])
    Wm = np.stack([2.0 + 3.0 * xi * np.ones(7) for xi in x])
    d = O.spline_derivs(x, Wm, np.ones(5, np.int32))
    assert np.allclose(d, 3.0, atol=1e-12)
    xref = np.linspace(0, 1, 5)
    out = O.spline_redist(x, xref, Wm, np.ones(5, np.int32), 1.0)
    assert np.allclose(out[1:-1], (2.0 + 3.0 * xref[1:-1])[:, None], atol=1e-12)
    assert np.array_equal(out[[0, -1]], Wm[[0, -1]])


def test_spline_natural_coefficients_by_hand():
    # natural spline through (0,0), (1,1), (2,0): c1 = -3/2 solves 4 c1 = 3(-1) - 3(1)
    c, b, d = O.spline_coeffs(np.array([0.0, 1.0, 2.0]), np.array([0.0, 1.0, 0.0]))
    assert np.allclose(c, [0.0, -1.5, 0.0])
    assert np.allclose(b[:2], [1.5, 0.0])
    assert np.allclose(d[:2], [-0.5, 0.5])


def _debye(f, x):
    """Debye function of a block of fraction f: 2 (f x + exp(-f x) - 1) / x^2."""
    return 2 * (f * x + np.exp(-f * x) - 1) / x**2


@pytest.mark.parametrize("f,L,ens", [(0.4, 3.0, 1), (0.5, 2.5, 1), (0.3, 4.0, 2), (0.45, 3.0, 2)])
def test_weak_single_mode_matches_rpa(f, L, ens):
    """Linear response of a pure diblock melt (phic = 1, so the homopolymer
    carries no weight) to W- = eps cos(2 pi x / L), W+ = 0: then wA = W- and
    wB = -W- (density.h:118-125), and the A density's cos mode is
    -(S_AA - S_AB) eps with the Debye functions S_AA = g(f), S_AB =
    (g(1) - g(f) - g(1 - f)) / 2 at x = k^2 / 6 (lengths in R0, diffusion
    exp(-k^2 ds / 6) per contour step, density.h:79-95).  The pseudo-spectral
    step is exact for one mode, so the oracle matches to about 1e-9."""
    m, N, eps = (32, 2, 2), 200, 1e-4
    D = np.array([L, 1.0, 1.0])
    M = int(np.prod(m))
    X = np.arange(m[0]) * L / m[0]
    w = np.zeros(6 * M)
    w[:M] = ((eps * np.cos(2 * np.pi * X / L))[:, None, None] * np.ones(m)).ravel()
    O.Density(m, D, N).props(w, N, 0.1, 1.0, f, ens)
    phiA = w[2 * M:3 * M].reshape(m)
    amp = 2 * np.mean(phiA[:, 0, 0] * np.cos(2 * np.pi * X / L))
    x = (2 * np.pi / L) ** 2 / 6
    fr = round(N * f) / N
    pred = -(_debye(fr, x) - 0.5 * (_debye(1, x) - _debye(fr, x) - _debye(1 - fr, x))) * eps
    assert abs(amp / pred - 1) <= 1e-6, (amp, pred)


@pytest.mark.parametrize("ens", [1, 2])
def test_richardson_step_is_fourth_order(ens):
    """Global convergence of lnQ in ds: the Richardson combination (4 S_half^2
    - S_full) / 3 (density.h:129-220) cancels the ds^2 error of the split
    step, so halving ds divides the error by 16.  Fields strong enough to
    matter (|W-| up to 5.5); n1 = N/2 and Nh = N/10 stay integers."""
    m, D = (16, 8, 8), np.array([3.0, 2.0, 2.0])
    M = int(np.prod(m))
    X = np.arange(m[0]) * D[0] / m[0]
    Y = np.arange(m[1]) * D[1] / m[1]
    wm = (4.0 * np.cos(2 * np.pi * X / D[0]))[:, None, None] + (1.5 * np.sin(2 * np.pi * Y / D[1]))[None, :, None] * np.ones(m)
    wp = (0.5 * np.cos(4 * np.pi * X / D[0]))[:, None, None] * np.ones(m)

    def lnq(N):
        w = np.zeros(6 * M)
        w[:M], w[M:2 * M] = wm.ravel(), wp.ravel()
        return O.Density(m, D, N).props(w, N, 0.1, 0.8, 0.5, ens)[0]

    ref = lnq(640)
    err = [abs(lnq(N) - ref) for N in (20, 40, 80, 160)]
    orders = [np.log2(err[i] / err[i + 1]) for i in range(3)]
    print("observed orders", orders)
    assert all(3.8 <= p <= 4.3 for p in orders), orders
