"""Boundary data / sources against independent numpy restatements, and the
manufactured Poisson pairs satisfy -Lap u = f (finite differences, FP64)."""
import numpy as np
import pytest


def charges_np(p, pts):
    q = np.array([[p.charges[k][j] for j in range(4)] for k in range(p.charge_count)], np.float64)
    d = pts[:, None, :] - q[None, :, :3]
    return (q[None, :, 3] / np.sqrt(np.maximum((d ** 2).sum(-1), 1e-12))).sum(1)


def test_seeded_charges_shell(n2w):
    p = n2w.problem_charges_seeded(8, 1.6, 2.0, 12345)
    q = np.array([[p.charges[k][j] for j in range(4)] for k in range(8)])
    r = np.linalg.norm(q[:, :3], axis=1)
    assert np.all((r >= 1.6 - 1e-5) & (r <= 2.0 + 1e-5))
    assert np.all(np.abs(q[:, 3]) <= 1.0)
    p2 = n2w.problem_charges_seeded(8, 1.6, 2.0, 12346)
    assert p2.charges[0][0] != p.charges[0][0]


def test_exact_and_f32_match_numpy(n2w):
    pts = np.random.default_rng(2).uniform(-1, 1, (300, 3))
    p = n2w.problem_charges_seeded()
    assert np.allclose(n2w.problem_exact(p, pts), charges_np(p, pts), rtol=1e-12)
    g, f = n2w.problem_eval_f32(p, pts)
    assert np.allclose(g, charges_np(p, pts), rtol=1e-5, atol=1e-6) and np.all(f == 0)
    w = 2 * np.pi * 1.5
    s = n2w.problem_sinprod(w)
    u = np.sin(w * pts[:, 0]) * np.sin(w * pts[:, 1]) * np.sin(w * pts[:, 2])
    assert np.allclose(n2w.problem_exact(s, pts), u, atol=1e-6)  # omega is stored as float32
    g, f = n2w.problem_eval_f32(s, pts)
    assert np.allclose(g, u, atol=1e-5) and np.allclose(f, 3 * w * w * u, rtol=1e-4, atol=1e-3)
    h = n2w.problem_reference(n2w.N2W_BC["harmonic_zebra_k8"])
    z = (pts[:, 0] + 1j * pts[:, 1]) ** 8
    assert np.allclose(n2w.problem_exact(h, pts), z.real, atol=1e-12)


@pytest.mark.parametrize("name", ["harmonic_x2_minus_y2", "external_charges_medium", "external_charges_high",
                                  "harmonic_zebra_k4", "harmonic_zebra_k12", "external_charges_shell_k8",
                                  "external_charges_shell_k16", "charges_seeded", "harmonic_mixture_smooth",
                                  "harmonic_mixture_figlike", "harmonic_mixture_multiscale",
                                  "harmonic_mixture_figlike_hf"])
def test_harmonic_modes_have_zero_laplacian(n2w, name):
    p = n2w.problem_from_name(name)
    pts = np.random.default_rng(3).uniform(-0.7, 0.7, (50, 3))
    h = 1e-3
    lap = -6 * n2w.problem_exact(p, pts)
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        lap += n2w.problem_exact(p, pts + e) + n2w.problem_exact(p, pts - e)
    lap /= h * h
    scale = np.abs(n2w.problem_exact(p, pts)).max() + 1
    assert np.abs(lap).max() < 2e-3 * scale * 100


@pytest.mark.parametrize("name", ["poisson_multiscale", "poisson_figlike_hf", "poisson_figlike_hf_x5",
                                  "poisson_sinprod"])
def test_poisson_pairs_satisfy_equation(n2w, name):
    p = n2w.problem_from_name(name)
    pts = np.random.default_rng(4).uniform(-0.7, 0.7, (40, 3))
    h = 1e-3
    lap = -6 * n2w.problem_exact(p, pts)
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        lap += n2w.problem_exact(p, pts + e) + n2w.problem_exact(p, pts - e)
    lap /= h * h
    _, f = n2w.problem_eval_f32(p, pts)
    assert np.allclose(-lap, f, rtol=2e-3, atol=2e-3 * (np.abs(f).max() + 1))


def test_mode_names_and_aliases(n2w):
    from n2w._lib import lib
    import ctypes as C

    for alias, mode in [("zebra8", 4), ("HARMONIC", 0), ("shell16", 7), ("const1", 12), ("poisson_hf", 31),
                        ("stripes_k8", 8), ("charges8_seeded", 100), ("sinprod", 101), ("fig4", 14),
                        ("hm_smooth", 13), ("multiscale", 15), ("fig_hf", 16), ("poisson", 30),
                        ("poisson_hf_x5", 32)]:
        m = C.c_int()
        assert lib.n2w_problem_mode_from_name(alias.encode(), C.byref(m)) == 0
        assert m.value == mode
    assert lib.n2w_problem_mode_name(4) == b"harmonic_zebra_k8"
    m = C.c_int()
    assert lib.n2w_problem_mode_from_name(b"nonsense", C.byref(m)) == 1


ANALYTIC_MODES = {13: "harmonic_mixture_smooth", 14: "harmonic_mixture_figlike", 15: "harmonic_mixture_multiscale",
                  16: "harmonic_mixture_figlike_hf", 30: "poisson_multiscale", 31: "poisson_figlike_hf",
                  32: "poisson_figlike_hf_x5"}


def check_against(n2w, mode, pts, u_ref, f_ref):
    p = n2w.problem_reference(mode)
    g, f = n2w.problem_eval_f32(p, pts)
    # FP32 evaluations of the same formulas: a few ulps of the term magnitudes apart
    np.testing.assert_allclose(g, u_ref, rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(f, f_ref, rtol=2e-5, atol=2e-5 * (np.abs(f_ref).max() + 1))
    ex = n2w.problem_exact(p, pts.astype(np.float64))
    np.testing.assert_allclose(ex, u_ref, rtol=2e-5, atol=2e-6)


@pytest.mark.parametrize("mode", sorted(ANALYTIC_MODES))
def test_analytic_modes_match_reference_golden(n2w, mode):
    """Boundary data u and source f of the reference's analytic modes against
    the reference's own header functions (golden vectors, tests/golden)."""
    from conftest import GOLDEN

    d = np.load(GOLDEN / "analytic_modes.npz")
    check_against(n2w, mode, d["points"], d[f"u_{mode}"], d[f"f_{mode}"])


@pytest.mark.parametrize("mode", sorted(ANALYTIC_MODES))
def test_analytic_modes_match_reference_live(n2w, mode):
    import oracle

    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    pts = np.random.default_rng(mode).uniform(-1.1, 1.1, (500, 3)).astype(np.float32)
    u, f = oracle.ref_analytic(mode, pts)
    check_against(n2w, mode, pts, u, f)
