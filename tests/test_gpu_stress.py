"""Box stress and parameter derivatives (no reference code): the adjoint
d lnQ/dL against central finite differences of the reference discretisation
(h = 1e-4, FP64), the FP32 adjoint against the FP64 adjoint, and dF/dL,
dF/dchiN at a converged saddle point against finite differences of
re-converged free energies."""
import numpy as np
import pytest

import scft_string_b200 as S

pytestmark = pytest.mark.gpu


def smooth_fields(m, D, seed, amp=3.0):
    rng = np.random.default_rng(seed)
    x = [np.arange(m[i]) * D[i] / m[i] for i in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    wm = amp * (np.cos(2 * np.pi * X / D[0]) + 0.5 * np.sin(2 * np.pi * Y / D[1]) * np.cos(2 * np.pi * Z / D[2]))
    wm += 0.2 * rng.normal(size=m)
    wp = 0.3 * rng.normal(size=m)
    return wm.ravel(), wp.ravel()


def lnq_at(ctx, D):
    ctx.set_box(D)
    ctx.props(0)
    return ctx.get_conc(0)[1]


@pytest.mark.parametrize("m,D,N,ens", [((8, 12, 10), (2.0, 3.0, 2.5), 20, 1),
                                        ((12, 8, 16), (3.1, 2.2, 4.0), 24, 2),
                                        ((32, 32, 32), (4.0, 4.0, 4.0), 40, 1)])
def test_adjoint_matches_finite_differences(built_lib, m, D, N, ens):
    D = np.array(D)
    wm, wp = smooth_fields(m, D, 1)
    ctx = S.Context(m, D, N, chi=12, f=0.45, phidb=0.8, ens=ens, alpha=0.1, strn=1, dostring=0)
    ctx.set_fields(0, wm, wp)
    dlnq, dF = ctx.stress(0)
    assert np.allclose(dF, -dlnq)
    h = 1e-4
    for i in range(3):
        Dp, Dm = D.copy(), D.copy()
        Dp[i] += h
        Dm[i] -= h
        fd = (lnq_at(ctx, Dp) - lnq_at(ctx, Dm)) / (2 * h)
        assert abs(dlnq[i] - fd) <= 1e-6 * max(1.0, abs(fd)), (i, dlnq[i], fd)
    ctx.set_box(D)
    # FP32 adjoint against the FP64 one
    c32 = S.Context(m, D, N, chi=12, f=0.45, phidb=0.8, ens=ens, alpha=0.1, strn=1, dostring=0,
                    precision="fp32")
    c32.set_fields(0, wm, wp)
    d32, _ = c32.stress(0)
    assert np.allclose(d32, dlnq, rtol=2e-4, atol=2e-6)


def converged(D, chi, m=(8, 8, 24), N=20):
    """Lamellar saddle point (z structure) to RMS residual 1e-10 by Anderson mixing."""
    D = np.asarray(D, float)
    ctx = S.Context(m, D, N, chi=chi, f=0.5, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0)
    z = np.arange(m[2]) * D[2] / m[2]
    wm = np.broadcast_to(0.4 * chi * np.cos(2 * np.pi * z / D[2]), m).ravel()
    ctx.set_fields(0, wm, np.zeros_like(wm))
    n, err = ctx.anderson_solve(0, maxIter=2000, tol=1e-10, nhist=12, lam=0.1)
    ctx.props(0)
    conc, lnQ, _ = ctx.get_conc(0)
    W = ctx.get_fields(0)
    M = ctx.M
    pA, pB = conc[:M], conc[M:2 * M]
    wa, wb = W[:M] + W[M:], W[M:] - W[:M]
    F = -lnQ + np.mean(chi * pA * pB - wa * pA - wb * pB)
    return ctx, F, err


def test_saddle_point_stress_and_dchi(built_lib):
    """At a converged saddle point the adjoint stress dF/dLz and the closed
    form dF/dchiN match central differences of re-converged free energies."""
    chi = 14.0
    D = np.array([2.0, 2.0, 4.6])
    ctx, F0, err = converged(D, chi)
    assert err <= 1e-10
    _, dF = ctx.stress(0)
    assert abs(dF[0]) < 1e-12 and abs(dF[1]) < 1e-12  # no x, y structure
    h = 1e-3
    _, Fp, ep = converged(D + [0, 0, h], chi)
    _, Fm, em = converged(D - [0, 0, h], chi)
    assert max(ep, em) <= 1e-10
    fd = (Fp - Fm) / (2 * h)
    print("dF/dLz adjoint", dF[2], "fd", fd)
    assert abs(dF[2] - fd) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
    dchi = ctx.dF_dchi(0)
    _, Fcp, _ = converged(D, chi + h)
    _, Fcm, _ = converged(D, chi - h)
    fdc = (Fcp - Fcm) / (2 * h)
    print("dF/dchi closed form", dchi, "fd", fdc)
    assert abs(dchi - fdc) <= 1e-6 * max(1.0, abs(fdc))


def test_variable_cell_relaxation_lowers_stress(built_lib):
    """A lamellar replica in a box longer than its period relaxes its cell:
    the adjoint stress falls below 1e-6 and the free energy does not rise."""
    m, N, chi = (8, 8, 24), 20, 14.0
    D = np.array([2.0, 2.0, 4.6])
    ctx = S.Context(m, D, N, chi=chi, f=0.5, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0)
    z = np.arange(m[2]) * D[2] / m[2]
    wm = np.broadcast_to(0.4 * chi * np.cos(2 * np.pi * z / D[2]), m).ravel()
    ctx.set_fields(0, wm, np.zeros_like(wm))
    ctx.solve_field0_all(5000, 1e-8)
    ctx.solve_field(150)
    _, s0 = ctx.stress(0)
    n, st, box = ctx.relax_cell(0, maxOuter=200, inner=15, stressTol=1e-6, gamma=2.0)
    print("rounds", n, "stress", st, "box", box, "initial stress", s0)
    assert np.abs(st).max() <= 1e-6
    assert abs(box[0] - D[0]) < 1e-12 and abs(box[1] - D[1]) < 1e-12  # no x, y structure: no stress


@pytest.mark.parametrize("m,D,N,ens,K,prec", [
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 1, 1, "fp64"),     # every slice a checkpoint
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 1, 3, "fp64"),     # K does not divide N
    ((12, 8, 16), (3.1, 2.2, 4.0), 24, 2, 5, "fp64"),
    ((12, 8, 16), (3.1, 2.2, 4.0), 24, 2, 100, "fp64"),   # one segment
    ((32, 32, 32), (4.0, 4.0, 4.0), 40, 1, 6, "fp64"),    # compile-time shape
    ((32, 32, 32), (4.0, 4.0, 4.0), 101, 1, 7, "fp32"),   # odd middle piece
    ((64, 64, 96), (4.2, 4.2, 6.3), 160, 1, 13, "fp32"),  # 64x64x96, N=160, every 13 steps
])
def test_checkpointed_adjoint_equals_full_store(built_lib, m, D, N, ens, K, prec):
    """The adjoint with propagators kept every K contour steps (recomputed in
    mirrored segment pairs) gives the full-store adjoint's values: the
    recomputed slices are the same bits, only the FP64 pair sums are added in
    another order."""
    D = np.array(D)
    wm, wp = smooth_fields(m, D, 2)
    ctx = S.Context(m, D, N, chi=12, f=0.45, phidb=0.8, ens=ens, alpha=0.1, strn=1, dostring=0,
                    precision=prec)
    ctx.set_fields(0, wm, wp)
    full, _ = ctx.stress(0)
    ck, dF, nbytes = ctx.stress_ckpt(0, K)
    assert np.allclose(dF, -ck)
    tol = 1e-11 * np.abs(full).max()
    assert np.abs(ck - full).max() <= tol, (ck, full)
    store = (N + 1) * 2 * ctx.M * (4 if prec == "fp32" else 8)
    if 3 <= K < N:
        assert nbytes < store
    print(m, N, K, prec, "checkpointed bytes", nbytes, "full store", store)
    # the full-store path still works after the checkpointed one reused slot 0
    again, _ = ctx.stress(0)
    np.testing.assert_array_equal(again, full)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_replica_boxes(built_lib, precision):
    """Every replica owns its box: replica 1 in a 2-replica context with its own
    box gives the densities and stress of a one-replica context in that box,
    bit for bit, while replica 0 keeps the common box."""
    m, N = (12, 8, 16), 24
    D0, D1 = np.array([3.1, 2.2, 4.0]), np.array([2.9, 2.4, 4.3])
    wm, wp = smooth_fields(m, D0, 3)
    two = S.Context(m, D0, N, chi=12, f=0.45, phidb=0.8, ens=1, alpha=0.1, strn=2, dostring=0,
                    precision=precision)
    one = S.Context(m, D1, N, chi=12, f=0.45, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0,
                    precision=precision)
    for ii in range(2):
        two.set_fields(ii, wm, wp)
    one.set_fields(0, wm, wp)
    two.set_box(D1, ii=1)
    np.testing.assert_array_equal(two.get_box(1), D1)
    np.testing.assert_array_equal(two.get_box(0), D0)
    two.props(1)
    one.props(0)
    c2, q2, _ = two.get_conc(1)
    c1, q1, _ = one.get_conc(0)
    assert q1 == q2
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(two.stress(1)[0], one.stress(0)[0])
    s0, _ = two.stress(0)
    ref = S.Context(m, D0, N, chi=12, f=0.45, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0,
                    precision=precision)
    ref.set_fields(0, wm, wp)
    np.testing.assert_array_equal(s0, ref.stress(0)[0])


@pytest.mark.parametrize("m,D,N,f,ens,K,prec,fcont", [
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.45, 1, 3, "fp64", 0),    # odd A block
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.45, 2, 1, "fp64", 0),    # every slice a checkpoint
    ((12, 8, 16), (3.1, 2.2, 4.0), 24, 0.43, 1, 5, "fp64", 1),    # junction step inside the chain
    ((32, 32, 32), (4.0, 4.0, 4.0), 40, 0.5, 2, 7, "fp32", 0),    # compile-time shape
    ((64, 64, 96), (4.2, 4.2, 6.3), 160, 0.4, 1, 13, "fp32", 0),  # 64x64x96, N=160, every 13 steps
])
def test_checkpointed_density_equals_props(built_lib, m, D, N, f, ens, K, prec, fcont):
    """The density pass from checkpoints (segments recomputed with their
    mirrors, Simpson terms accumulated per point) gives the densities, lnQ and
    phis of the full-store props: the slices are the same bits, only the FP64
    sums run in another order."""
    D = np.array(D)
    wm, wp = smooth_fields(m, D, 4)
    ctx = S.Context(m, D, N, chi=12, f=f, phidb=0.8, ens=ens, alpha=0.1, strn=1, dostring=0,
                    precision=prec, fcont=fcont)
    ctx.set_fields(0, wm, wp)
    ctx.props(0)
    c0, q0, p0 = ctx.get_conc(0)
    q1, p1, nbytes = ctx.props_ckpt(0, K)
    c1, q2, p2 = ctx.get_conc(0)
    assert q1 == q2 and np.array_equal(p1, p2)
    assert abs(q1 - q0) <= 1e-13 * abs(q0)
    np.testing.assert_allclose(p1, p0, rtol=1e-12, atol=1e-15)
    assert np.abs(c1 - c0).max() <= 1e-12 * np.abs(c0).max()
    store = (N + 1) * 2 * ctx.M * (4 if prec == "fp32" else 8)
    if 3 <= K < N:
        assert nbytes < store + 6 * 8 * ctx.M
    print(m, N, K, prec, "checkpointed density bytes", nbytes, "full store", store)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_context_without_full_store(built_lib, precision):
    """nostore: every props runs from checkpoints, so the W+ prelude and the
    string iterations follow the full-store run (the same densities up to the
    order of the FP64 sums); the box stress comes from the checkpointed
    adjoint; the calls that read the store refuse."""
    from scft_string_b200.configs import STRING_64, fields
    c = dict(STRING_64, m=(16, 16, 16), D=(2.5, 2.5, 2.5), N=24, strn=4)
    wm, wp = fields(c)
    runs = []
    for nostore in (0, 1):
        ctx = S.StringSolver(dict(c, nostore=nostore, ckpt_K=5), precision=precision)
        for ii in range(c["strn"]):
            ctx.set_fields(ii, wm[ii], wp[ii])
        ctx.solve_field0_all(50, 1e-6)
        ctx.string_begin(100, 1e-3)
        errs = [ctx.string_step()["errtot"] for _ in range(4)]
        W = np.stack([ctx.get_fields(ii) for ii in range(c["strn"])])
        st = ctx.stress(1)[1]
        runs.append((errs, W, st, ctx))
    (e0, W0, s0, _), (e1, W1, s1, ctx1) = runs
    np.testing.assert_allclose(e1, e0, rtol=1e-9)
    assert np.abs(W1 - W0).max() <= 1e-9 * np.abs(W0).max()
    np.testing.assert_allclose(s1, s0, rtol=1e-7, atol=1e-12)
    with pytest.raises(S.ScftError):
        ctx1.do_step(0, np.ones(2 * ctx1.M), 0)
    with pytest.raises(S.ScftError):
        ctx1.propagator(0, 0, 1)


@pytest.mark.parametrize("m,D,N,ens", [((8, 12, 10), (2.0, 3.0, 2.5), 20, 1),
                                        ((12, 8, 16), (3.1, 2.2, 4.0), 24, 2),
                                        ((32, 32, 32), (4.0, 4.0, 4.0), 24, 1)])
def test_adjoint_matches_the_oracle(built_lib, m, D, N, ens):
    """The CUDA adjoint (Parseval sums of the FFT'd operands) against the
    oracle's FP64 restatement (oc_stress: dS/dL applied in real space) at the
    same fields: the full-store and the checkpointed FP64 adjoint to 1e-10,
    the FP32 one within the FP32 bound of the finite-difference test."""
    import oracle as O
    D = np.array(D)
    wm, wp = smooth_fields(m, D, 5)
    f = round(N * 0.45) / N
    ref = O.Density(m, D, N).stress(np.concatenate([wm, wp]), N, 0.1, 0.8, f, ens)
    for prec in ("fp64", "fp32"):
        ctx = S.Context(m, D, N, chi=12, f=0.45, phidb=0.8, ens=ens, alpha=0.1, strn=1, dostring=0,
                        precision=prec)
        ctx.set_fields(0, wm, wp)
        full, _ = ctx.stress(0)
        ck, _, _ = ctx.stress_ckpt(0, 5)
        if prec == "fp64":
            assert np.abs(full - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max()), (full, ref)
            assert np.abs(ck - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max()), (ck, ref)
        else:
            assert np.allclose(full, ref, rtol=2e-4, atol=2e-6), (full, ref)
