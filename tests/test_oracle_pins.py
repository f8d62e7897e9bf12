"""Known answers the reference's own tests hold, pinned on the oracle (CPU).

- Si (222), 30 keV electron along z, photon at 100 deg in the x-z plane at
  the exact vacuum root: the second-order PXR and CBS line elements of both
  polarisations, quantum (h = hbar c / m c^2) and classical (h = 0), from an
  independent 60-digit evaluation quoted in the reference's
  ``tests/montecarlo/spectrum/test_quantum_cb_elements.py:85-116``.
- h -> 0 gives the classical braced form (the same file, ``:53-61``): here
  restated from the classical PXR numerator (v.g + k.v)(g.e + k.e) - k^2 (v.e)
  and the CBS element -[(g.e - (v.g)(v.e)) + (v.e)(k.g - (k.v)(v.g))/(v.g)] / (gamma v.g).
"""

import numpy as np

import oracle

MC2_EV = 510998.95
H = 1973.269804 / MC2_EV  # hbar c / m c^2 [Angstrom]

# 60-digit values rounded to FP64: the vacuum root omega [1/Angstrom] and, for
# sigma then pi, ((pxr_num, f_cbs) quantum, (pxr_num, f_cbs) classical).
SI222_OMEGA = 0.68665746147068140754
SI222 = (
    ((1.5907956780189942, -2.9955100457228503), (1.6674555552543886, -2.876417643261264)),
    ((1.690198839167976, -3.9242147431280814), (1.7791971109401228, -3.724387851171339)),
)


def _factors(h, gamma, v, g, k, e):
    return oracle.quantum_line_factors(h, gamma, v @ g, k @ v, k @ g, g @ g, k @ k, v @ e, g @ e, k @ e)


def test_si222_30kev_sixty_digit_pin():
    gamma = 1.0 + 3e4 / MC2_EV
    v = np.array([0.0, 0.0, np.sqrt(1.0 - 1.0 / gamma ** 2)])
    g = np.full(3, 4.0 * np.pi / 5.431)
    th = np.radians(100.0)
    n = np.array([np.sin(th), 0.0, np.cos(th)])
    k = SI222_OMEGA * n
    e_sigma = np.array([0.0, 1.0, 0.0])
    for e, (quantum, classical) in zip((e_sigma, np.cross(n, e_sigma)), SI222, strict=True):
        np.testing.assert_allclose(_factors(H, gamma, v, g, k, e), quantum, rtol=1e-12)
        np.testing.assert_allclose(_factors(0.0, gamma, v, g, k, e), classical, rtol=1e-12)
    # sigma is perpendicular to v and k: the classical CBS element is -(g.e)/(gamma v.g)
    np.testing.assert_allclose(SI222[0][1][1], -(g @ e_sigma) / (gamma * (v @ g)), rtol=1e-12)


def test_classical_limit_is_the_braced_form():
    rng = np.random.default_rng(0)
    for _ in range(200):
        T = 1e5 * rng.random() + 1e3
        gamma = 1.0 + T / MC2_EV
        v = rng.normal(size=3)
        v *= np.sqrt(1.0 - 1.0 / gamma ** 2) / np.linalg.norm(v)
        g = rng.normal(size=3) * 3.0
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        k = (0.05 + rng.random()) * n
        e = np.cross(n, rng.normal(size=3))
        e /= np.linalg.norm(e)
        vdg, kv, kg, ve = v @ g, k @ v, k @ g, v @ e
        pxr0 = (vdg + kv) * (g @ e + k @ e) - (k @ k) * ve
        cbs0 = -((g @ e - vdg * ve) + ve * (kg - kv * vdg) / vdg) / (gamma * vdg)
        np.testing.assert_allclose(_factors(0.0, gamma, v, g, k, e), [pxr0, cbs0], rtol=1e-12)


def test_segment_mean_transmission_against_quadrature():
    """Segment mean of exp(-tau) for tau linear along the segment, against
    adaptive quadrature at the reference's own test points, including the
    equal-depth and near-equal limits and a tau of 800
    (tests/montecarlo/spectrum/test_segment_escape.py:54-72)."""
    from scipy.integrate import quad

    tau0 = [0.0, 0.3, 2.0, 5.0, 40.0, 1.0]
    tau1 = [0.0, 0.3 + 1e-6, 0.5, 9.0, 800.0, 1.0 + 3e-5]
    for a, b in zip(tau0, tau1):
        ref = quad(lambda s: np.exp(-(a + (b - a) * s)), 0.0, 1.0, epsabs=0.0, epsrel=1e-13)[0]
        got = oracle.mean_transmission(a, b)
        assert abs(got - ref) <= 1e-9 * ref
        assert oracle.mean_transmission(b, a) == got
        assert got <= np.exp(-min(a, b))
    assert oracle.mean_transmission(0.0, 0.0) == 1.0


def test_node_reducer_matches_the_dense_sinc_squared_contraction():
    """spec += sum_j w_j sinc^2(a_j (E - E_j)) against the dense matrix form,
    with an exact resonance on a node (the x = 0 guard) and empty input
    leaving the spectrum unchanged (tests/montecarlo/transport/test_cxr_cpu_reduce.py)."""
    rng = np.random.default_rng(7)
    E_grid = np.linspace(1000.0, 20000.0, 97)
    E_r = rng.uniform(900.0, 20100.0, 513)
    E_r[0] = E_grid[11]
    a = rng.uniform(1.0e-3, 0.5, E_r.size)
    w = rng.random(E_r.size)
    x = a[:, None] * (E_grid[None, :] - E_r[:, None])
    S = np.where(x == 0.0, 1.0, np.sin(np.where(x == 0.0, 1.0, x)) / np.where(x == 0.0, 1.0, x)) ** 2
    np.testing.assert_allclose(oracle.reduce_node(E_r, a, w, E_grid), w @ S, rtol=1e-12, atol=0.0)
    assert np.array_equal(oracle.reduce_node(np.empty(0), np.empty(0), np.empty(0), E_grid), np.zeros(E_grid.size))
