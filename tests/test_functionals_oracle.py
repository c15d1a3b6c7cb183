"""The functionals of alsfvm/src/functional/ in the oracle (CPU).

Identity, Moment, LogEntropy, BoundedVariation, Legendre and
LegendrePointWise are pinned bit for bit to the reference's own classes:
their sources are compiled into the reference build (oracle/_ref, with a
property-tree stand-in for their parameters) and made by name through its
FunctionalFactory; the committed fixture tests/golden/functionals_ref.npz
carries their outputs where that build is absent.  The Legendre classes
call boost::math::legendre_p, which is not in this image: the build gets a
restatement of it (oracle/ref_shims/boost/math/special_functions/
legendre.hpp: long double evaluation, negative degrees reflected, a domain
error outside [-1, 1], as Boost's default policy has it), so what these
fixtures pin is the reference's use of it (scaling, midpoints, sums,
weights).  The restatement is also checked against the reference's own
unit tests (test/library_tests/src/fvm/functional/EntropyTest.cpp,
LegendreTest.cpp), ported with their inputs and tolerances, and against
SciPy's Legendre polynomials.  The alsuq statistics bv_direction and
structure_2pt are checked against direct NumPy evaluations of their stated
formulas.
"""
import os

import numpy as np
import pytest
import scipy.special

from oracle_lib import padded_shape, smooth_random_state

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

GAMMA = 1.4


def _midpoints(n, lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0)):
    """Cell midpoints origin + dx*i + dx/2 (Grid.cpp:148-171)."""
    return [lower[d] + (upper[d] - lower[d]) / n[d] * np.arange(n[d]) +
            (upper[d] - lower[d]) / n[d] / 2.0 for d in range(len(n))]


def _euler2_state(n, g, E_of):
    """fill_volume with rho = e, m_x = m_y = sin(2 pi x y) at the midpoints."""
    shp = padded_shape(2, n, g)
    U = np.zeros(shp)
    x, y = _midpoints(n)
    X, Y = np.meshgrid(x, y)
    rho = np.full_like(X, np.exp(1.0))
    m = np.sin(2 * np.pi * X * Y)
    U[0, 0, g:-g, g:-g] = rho
    U[1, 0, g:-g, g:-g] = m
    U[2, 0, g:-g, g:-g] = m
    U[3, 0, g:-g, g:-g] = E_of(rho, m)
    return U


def test_log_entropy_result_is_zero(c_oracle):
    """EntropyTest.ResultIsZeroTest: p = e^1.4, rho = e, so s = 0."""
    n, g = (3, 2), 2
    U = _euler2_state(n, g, lambda rho, m: np.exp(1.4) / 0.4 + .5 * (2 * m * m) / rho)
    out = c_oracle.functional(2, n, g, "log_entropy", U, weight=0.5, gamma=GAMMA)
    assert abs(out[3, 0]) < 1e-8


def test_log_entropy_result_is_one(c_oracle):
    """EntropyTest.ResultIsOneTest: s = 0.4/e, so -rho s/(gamma-1) = -1 on
    the unit square; weight -1 gives 1."""
    n, g = (2, 2), 2
    U = _euler2_state(n, g, lambda rho, m: np.exp(1.4 + 0.4 / np.exp(1)) / 0.4 +
                      .5 * (2 * m * m) / rho)
    out = c_oracle.functional(2, n, g, "log_entropy", U, weight=-1.0, gamma=GAMMA)
    assert abs(out[3, 0] - 1.0) < 1e-8
    assert np.all(out[:3] == 0)


def test_legendre_constant(c_oracle):
    """LegendreTest.ConstantTest: every variable sin(2 pi x y) at the
    midpoints, degrees 0, range [-1, 1], weight 0.5 -> 0.5 per variable
    (ASSERT_DOUBLE_EQ: within 4 ulps)."""
    n, g = (3, 2), 2
    U = np.zeros(padded_shape(2, n, g))
    x, y = _midpoints(n)
    X, Y = np.meshgrid(x, y)
    U[:, 0, g:-g, g:-g] = np.sin(2 * np.pi * X * Y)[None]
    out = c_oracle.functional(2, n, g, "legendre", U, weight=0.5, degree_k=0, degree_n=0,
                              degree_m=0, min_value=-1, max_value=1)
    assert np.all(np.abs(out[:, 0] - 0.5) <= 4 * np.spacing(0.5))


@pytest.mark.parametrize("degree", range(12))
def test_legendre_polynomials_against_scipy(c_oracle, degree):
    """P_degree(u) through legendre_pointwise (min 0, max 1: the value is u)
    against scipy.special.eval_legendre on [-1, 1]."""
    n, g = (21, 5), 1
    u = np.linspace(-1, 1, 21)
    U = np.zeros(padded_shape(2, n, g))
    U[:, 0, g:-g, g:-g] = u[None, None, :]
    out = c_oracle.functional(2, n, g, "legendre_pointwise", U, degree=degree, min_value=0.0,
                              max_value=1.0)
    ref = scipy.special.eval_legendre(degree, u)
    np.testing.assert_allclose(out[0].reshape(5, 21), np.broadcast_to(ref, (5, 21)), rtol=0,
                               atol=1e-14)


def test_legendre_integral_formula(c_oracle):
    """legendre: sum over cells of P_k(x') P_n(y') P_m(u') dV with x', y' the
    midpoints scaled to [-1, 1] and u' = (u - min)/(max - min)."""
    n, g = (9, 7), 2
    st = smooth_random_state(21, 2, n, g)
    out = c_oracle.functional(2, n, g, "legendre", st, weight=1.5, degree_k=2, degree_n=3,
                              degree_m=1, min_value=-3.0, max_value=3.0)
    x, y = _midpoints(n)
    X, Y = np.meshgrid(2 * x - 1, 2 * y - 1)
    for v in range(4):
        val = (st[v, 0, g:-g, g:-g] + 3.0) / 6.0
        ref = np.sum(scipy.special.eval_legendre(2, X) * scipy.special.eval_legendre(3, Y) *
                     val) * (1 / 9) * (1 / 7)
        assert abs(out[v, 0] - 1.5 * ref) < 1e-13


@pytest.mark.parametrize("dim,n", [(1, (17,)), (2, (9, 8)), (3, (5, 6, 4))])
def test_identity_and_moment(c_oracle, dim, n):
    g = 2
    st = smooth_random_state(31 + dim, dim, n, g)
    ident = c_oracle.functional(dim, n, g, "identity", st, weight=0.25)
    sl = tuple([slice(None)] + [slice(g, -g) if 3 - a <= dim else slice(None) for a in range(3)])
    np.testing.assert_array_equal(ident, 0.25 * st[sl].reshape(dim + 2, -1))
    mom = c_oracle.functional(dim, n, g, "moment", st, weight=2.0, degree=3)
    np.testing.assert_allclose(mom, 2.0 * st.reshape(dim + 2, -1) ** 3, rtol=1e-15)


@pytest.mark.parametrize("dim,n", [(1, (17,)), (2, (9, 8))])
@pytest.mark.parametrize("p", [1, 2])
def test_bounded_variation(c_oracle, dim, n, p):
    """sum over interior cells after the first along x (and y) of
    |(u - u_below, u - u_left)|^p (HostMemory::getTotalVariation)."""
    g = 2
    st = smooth_random_state(41 + dim, dim, n, g)
    out = c_oracle.functional(dim, n, g, "bv", st, weight=1.0, degree=p)
    for v in range(dim + 2):
        if dim == 1:
            u = st[v, 0, 0, g:-g]
            ref = np.sum(np.abs(np.diff(u)) ** p)
        else:
            u = st[v, 0, g:-g, g:-g]
            dx = u[1:, 1:] - u[1:, :-1]
            dy = u[1:, 1:] - u[:-1, 1:]
            ref = np.sum(np.sqrt(dx * dx + dy * dy) ** p)
        assert abs(out[v, 0] - ref) < 1e-12 * max(1.0, abs(ref))


def test_log_entropy_formula_3d(c_oracle):
    n, g = (6, 5, 4), 2
    st = smooth_random_state(51, 3, n, g)
    out = c_oracle.functional(3, n, g, "log_entropy", st, weight=1.0, gamma=GAMMA,
                              upper=(2.0, 1.0, 0.5))
    U = st[:, g:-g, g:-g, g:-g]
    msq = U[1] ** 2 + U[2] ** 2 + U[3] ** 2
    p = (GAMMA - 1) * (U[4] - msq / (2 * U[0]))
    s = np.log(p) - GAMMA * np.log(U[0])
    ref = np.sum(-U[0] * s / (GAMMA - 1)) * (2.0 / 6) * (1.0 / 5) * (0.5 / 4)
    assert abs(out[4, 0] - ref) < 1e-12 * abs(ref)


def test_legendre_needs_two_dimensions(c_oracle):
    st = smooth_random_state(1, 1, (8,), 1)
    with pytest.raises(ValueError):
        c_oracle.functional(1, (8,), 1, "legendre", st)


@pytest.mark.parametrize("dim,n,direction", [(1, (17,), 0), (2, (9, 8), 1), (3, (5, 6, 4), 2)])
def test_bv_direction(c_oracle, dim, n, direction):
    """alsuq bv_direction: sum of |u(x) - u(x - e_d)|^p from one cell after
    the start along d."""
    g = 2
    st = smooth_random_state(71 + dim, dim, n, g)
    out = c_oracle.functional(dim, n, g, "bv_direction", st, degree=2, direction=direction)
    sl = tuple([slice(None)] + [slice(g, -g) if 3 - a <= dim else slice(None) for a in range(3)])
    U = st[sl]
    axis = 3 - direction
    for v in range(dim + 2):
        ref = np.sum(np.abs(np.diff(U[v], axis=axis - 1)) ** 2)
        assert abs(out[v, 0] - ref) < 1e-12 * ref


def test_structure_two_points(c_oracle):
    """alsuq structure_2pt: (u(x+h1 e)-u)^2 (u(x+h2 e)-u) / cells summed,
    shifts clamped at the last cell, h1 fastest."""
    dim, n, g, H = 2, (11, 7), 2, 4
    st = smooth_random_state(81, dim, n, g)
    out = c_oracle.functional(dim, n, g, "structure_2pt", st, direction=0, number_of_h=H)
    for v in range(4):
        u = st[v, 0, g:-g, g:-g]
        ref = np.zeros((H, H))
        for h1 in range(H):
            i1 = np.minimum(np.arange(n[0]) + h1, n[0] - 1)
            for h2 in range(H):
                i2 = np.minimum(np.arange(n[0]) + h2, n[0] - 1)
                ref[h2, h1] = np.sum((u[:, i1] - u) ** 2 * (u[:, i2] - u)) / (n[0] * n[1])
        np.testing.assert_allclose(out[v].reshape(H, H), ref, rtol=1e-12, atol=1e-16)


def _fixture_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden",
                                                  os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


MG = _fixture_cases()


@pytest.mark.parametrize("dim,n,kind,degree", MG.FUNCTIONAL_CASES,
                         ids=[MG.functional_case_name(c[0], c[2], c[3])
                              for c in MG.FUNCTIONAL_CASES])
def test_functionals_equal_reference_fixture(c_oracle, dim, n, kind, degree):
    """The restatement gives the reference classes' bits (fixture made by
    the reference build's FunctionalFactory)."""
    z = np.load(os.path.join(GOLDEN, "functionals_ref.npz"))
    name = MG.functional_case_name(dim, kind, degree)
    for k in range(MG.FUNCTIONAL_MEMBERS):
        st = smooth_random_state(600 + 7 * k + dim, dim, n, 2)
        got = c_oracle.functional(dim, n, 2, kind, st, weight=MG.FUNCTIONAL_WEIGHT,
                                  out=z[name + "/start"][k], degree=degree, gamma=GAMMA,
                                  lower=MG.FUNCTIONAL_BOX[0], upper=MG.FUNCTIONAL_BOX[1])
        np.testing.assert_array_equal(got, z[name + "/result"][k])


@pytest.mark.parametrize("kind,params", MG.LEGENDRE_CASES,
                         ids=[MG.legendre_case_name(*c) for c in MG.LEGENDRE_CASES])
def test_legendre_equal_reference_fixture(c_oracle, kind, params):
    """Legendre and LegendrePointWise of the reference build (with Boost's
    legendre_p restated) give the same bits as the oracle."""
    z = np.load(os.path.join(GOLDEN, "functionals_ref.npz"))
    name = MG.legendre_case_name(kind, params)
    lo, hi = MG.LEGENDRE_RANGE
    for k in range(MG.FUNCTIONAL_MEMBERS):
        st = smooth_random_state(600 + 7 * k + 2, 2, MG.LEGENDRE_N, 2)
        got = c_oracle.functional(2, MG.LEGENDRE_N, 2, kind, st, weight=MG.FUNCTIONAL_WEIGHT,
                                  out=z[name + "/start"][k], min_value=lo, max_value=hi,
                                  lower=MG.FUNCTIONAL_BOX[0], upper=MG.FUNCTIONAL_BOX[1],
                                  **params)
        np.testing.assert_array_equal(got, z[name + "/result"][k])


@pytest.mark.parametrize("seed", range(4))
def test_legendre_equal_reference_build(c_oracle, ref_oracle, seed):
    """Fresh random Legendre cases against the reference build itself
    (skipped where it is not built), negative degrees included."""
    rng = np.random.default_rng(40 + seed)
    n = tuple(int(v) for v in rng.integers(4, 12, 2))
    g = int(rng.integers(1, 4))
    st = smooth_random_state(740 + seed, 2, n, g)
    lo, hi = tuple(rng.uniform(-1, 0, 3)), tuple(rng.uniform(1, 2, 3))
    w = float(rng.uniform(-2, 2))
    vrange = dict(min_value=-4.0 + seed, max_value=4.0 + seed)
    for kind, params in (("legendre", dict(degree_k=int(rng.integers(0, 6)),
                                           degree_n=int(rng.integers(-4, 6)),
                                           degree_m=int(rng.integers(0, 9)))),
                         ("legendre_pointwise", dict(degree=int(rng.integers(-6, 12))))):
        ref = ref_oracle.functional(2, n, g, kind, st, weight=w, lower=lo, upper=hi,
                                    **vrange, **params)
        got = c_oracle.functional(2, n, g, kind, st, weight=w, lower=lo, upper=hi,
                                  **vrange, **params)
        np.testing.assert_array_equal(got, ref)


def test_legendre_domain_and_negative_degrees(c_oracle):
    """Boost's legendre_p, as the reference calls it: an argument outside
    [-1, 1] is a domain error, and degree -l - 1 is degree l."""
    n, g = (6, 5), 2
    st = smooth_random_state(3, 2, n, g)
    with pytest.raises(ValueError, match="outside"):
        c_oracle.functional(2, n, g, "legendre_pointwise", st, degree=2, min_value=0.9,
                            max_value=1.1)
    for l in range(6):
        a = c_oracle.functional(2, n, g, "legendre_pointwise", st, degree=l, min_value=-3,
                                max_value=3)
        b = c_oracle.functional(2, n, g, "legendre_pointwise", st, degree=-l - 1, min_value=-3,
                                max_value=3)
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("kind", ["identity", "moment", "log_entropy", "bv"])
def test_functionals_equal_reference_build(c_oracle, ref_oracle, kind, seed):
    """Fresh random cases against the reference build itself (skipped where
    it is not built): grids, degrees, weights and boxes vary with the seed."""
    rng = np.random.default_rng(seed)
    dim = int(rng.integers(1, 3 if kind == "bv" else 4))
    n = tuple(int(v) for v in rng.integers(4, 12, dim))
    g = int(rng.integers(1, 4))
    degree = int(rng.integers(1, 4))
    lo = tuple(rng.uniform(-1, 0, 3))
    hi = tuple(rng.uniform(1, 2, 3))
    st = smooth_random_state(700 + seed, dim, n, g)
    w = float(rng.uniform(-2, 2))
    ref = ref_oracle.functional(dim, n, g, kind, st, weight=w, degree=degree, gamma=GAMMA,
                                lower=lo, upper=hi)
    got = c_oracle.functional(dim, n, g, kind, st, weight=w, degree=degree, gamma=GAMMA,
                              lower=lo, upper=hi)
    np.testing.assert_array_equal(got, ref)


def test_meanvar_statistics_by_name_equal_fixture(ref_oracle):
    """alsuq's MeanVariance made by name through its StatisticsFactory and
    run like the UQ runner (combine, finalize, write) gives the fixture's bits."""
    z = np.load(os.path.join(GOLDEN, "meanvar_7.npz"))
    states = np.stack([smooth_random_state(int(s), 2, (6, 5), 2) for s in z["seeds"]])
    mean, var = ref_oracle.statistics(2, (6, 5), 2, states, platform="cpu", name="meanvar")
    np.testing.assert_array_equal(mean, z["mean"])
    np.testing.assert_array_equal(var, z["var"])
