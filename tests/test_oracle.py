"""The oracle pinned against the reference's own golden vectors and, when built, against the reference itself."""
import numpy as np
import pytest

from compare import match_rows, theta_to_degrees
from conftest import GAUSS_PARAMS


@pytest.mark.parametrize("watershed", [True, False])
@pytest.mark.parametrize("fit", [0, 1, 2, 3, 4])
def test_oracle_matches_golden_csv(orc, stacks, goldens, fit, watershed):
    # Tests_CPU/test_Palm.cpp:236-249: stack.tif, thr 103.6, roi 7, sigma 1/2, ratio 0 (watershed) or 10
    rows = orc.localization(stacks["stack"], 103.6, 0.0 if watershed else 10.0, fit, GAUSS_PARAMS)
    key = "stack-localizations-103.6_%s_%d_1.0_0.0_7" % (watershed, fit)
    bad, worst, _ = match_rows(theta_to_degrees(rows, fit), goldens[key], atol=1e-3, rtol=1e-5)
    assert bad == 0, (key, worst)


def test_oracle_quadrants(orc, stacks, goldens):
    # Tests_CPU/test_Palm.cpp:252-264
    rows = orc.localization(stacks["stack_quadrant"], 103.6, 0.0, 4, GAUSS_PARAMS)
    bad, worst, _ = match_rows(theta_to_degrees(rows, 4), goldens["stack_quadrant-localizations-103.6_True_4_1.0_0.0_7"])
    assert bad == 0, worst


@pytest.mark.parametrize("fit", [0, 1, 2, 3, 4])
def test_oracle_first_plane_golden(orc, stacks, goldens, fit):
    rows = orc.localization(stacks["stack"][:1], 103.6, 0.0, fit, GAUSS_PARAMS)
    bad, worst, _ = match_rows(theta_to_degrees(rows, fit), goldens["stack-localizations-0_103.6_True_%d_1.0_0.0_7" % fit])
    assert bad == 0, worst


def test_oracle_plane_selection_golden(orc, stacks, goldens):
    rows = orc.localization(stacks["stack"][2:7], 103.6, 0.0, 4, GAUSS_PARAMS)
    rows[:, 1] += 2
    bad, worst, _ = match_rows(theta_to_degrees(rows, 4), goldens["stack-localizations-plane_select-103.6_True_4_1.0_0.0_7"])
    assert bad == 0, worst


@pytest.mark.parametrize("plane", range(10))
def test_oracle_auto_threshold(orc, stacks, plane):
    # Tests_CPU/test_Palm.cpp:305-321 (tolerance 1e-5)
    t = orc.auto_threshold(stacks["stack"][plane], np.array([7.0]))
    assert abs(t - stacks["auto_threshold"][plane]) < 1e-5


def test_oracle_atrous_identities(orc):
    # Tests_CPU/test_loc_ATrous.cpp: planes sum to the input; constant images have zero details
    for h, w in [(1, 1), (1, 9), (9, 1), (7, 13)]:
        img = ((np.arange(h * w) * 37 + 11) % 4096).astype(np.uint16).reshape(h, w)
        pl = orc.planes(img)
        assert np.allclose(pl.sum(axis=0), img, atol=1e-10)
    for v in (0, 1, 1024, 65535):
        pl = orc.planes(np.full((7, 11), v, dtype=np.uint16))
        assert np.all(pl[0] == 0) and np.all(pl[1] == 0) and np.all(pl[2] == v)


def test_oracle_segmentation_cases(orc):
    # Tests_CPU/test_loc_Segmentation2D.cpp:173-287 (strict threshold, surface > 4, connected peaks, absorbed peak)
    pot = np.zeros((5, 7))
    pot[1:4, 2:5] = 10
    assert len(orc.candidates_from_potential(pot, 9.0, 0)) == 1
    assert len(orc.candidates_from_potential(pot, 10.0, 0)) == 0
    for length, expect in [(3, 0), (4, 0), (5, 1)]:
        pot = np.zeros((5, 9))
        pot[2, 1:1 + length] = 10
        assert len(orc.candidates_from_potential(pot, 0, 0)) == expect
    for merge in (True, False):
        for first_higher in (True, False):
            pot = np.zeros((7, 13))
            pot[2:5, 2:5] = 100 if first_higher else 60
            pot[2:5, 8:11] = 60 if first_higher else 100
            pot[3, 5] = 40 if first_higher else 30
            pot[3, 6] = 20
            pot[3, 7] = 30 if first_higher else 40
            c = orc.candidates_from_potential(pot, 0, 10 if merge else 0)
            assert len(c) == (1 if merge else 2)
            assert c[:, 3].sum() == 21 and c[:, 2].sum() == pot.sum()
    pot = np.zeros((7, 18))
    pot[2:5, 1:4] = 200
    pot[2:5, 7:10] = 100
    pot[2:5, 13:16] = 60
    pot[3, 10], pot[3, 11], pot[3, 12] = 40, 20, 30
    c = orc.candidates_from_potential(pot, 0, 10)
    assert len(c) == 2 and c[0, 3] == 9 and c[0, 2] == 1800 and c[1, 3] == 21 and c[1, 2] == 1530


def test_oracle_many_regions(orc):
    # Tests_CPU/test_loc_Segmentation2D.cpp: labels beyond 16 bits
    pot = np.zeros((1025, 1025))
    for y in range(1, 1024, 4):
        for x in range(1, 1024, 4):
            pot[y:y + 3, x:x + 3] = 100
    c = orc.candidates_from_potential(pot, 0, 0)
    assert len(c) == 65536 and np.all(c[:, 3] == 9) and np.all(c[:, 2] == 900)


def test_oracle_equals_reference_build(orc, ref, stacks):
    """Bit-for-bit against the reference compiled from its own sources (skipped where oracle/_ref is absent)."""
    if ref is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    import synth
    s, _ = synth.stack("c1", frames=6, seed=5)
    thr = synth.mad_threshold(orc.planes(s[0])[1])
    for stack, t in ((stacks["stack"], 103.6), (s, thr)):
        for ratio in (0.0, 10.0):
            for fit in range(5):
                a = orc.localization(stack, t, ratio, fit, GAUSS_PARAMS)
                b = ref.localization(stack, t, ratio, fit, GAUSS_PARAMS)
                assert a.shape == b.shape and np.array_equal(a, b), (fit, ratio)
        assert np.array_equal(orc.wavelett(stack, 2), ref.wavelett(stack, 2))
        for k in range(stack.shape[0]):
            assert np.array_equal(orc.candidates(stack[k], t, 10.0), ref.candidates(stack[k], t, 10.0))
    rows = ref.localization(stacks["stack"], 103.6, 0.0, 0, GAUSS_PARAMS)
    pos = np.stack([rows[:, 0], rows[:, 1], rows[:, 4], rows[:, 5], rows[:, 15], rows[:, 16]], axis=1)
    for fit in (1, 2, 3, 4):
        assert np.array_equal(orc.fitting(stacks["stack"], pos, fit, GAUSS_PARAMS), ref.fitting(stacks["stack"], pos, fit, GAUSS_PARAMS))


def test_oracle_spline_equals_reference_build(orc, ref, stacks):
    if ref is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    import spline_table
    for roi, dist in ((7, 0.0), (13, 0.3)):
        params = spline_table.fit_params(roi=roi, sx=15, sy=15, sz=31, dz_nm=30.0, distortion=dist, seed=2)
        a = orc.localization(stacks["stack"][:4], 103.6, 0.0, 5, params)
        b = ref.localization(stacks["stack"][:4], 103.6, 0.0, 5, params)
        assert a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


# ---- Astigmatism3DEstimation (AstigFit::Estimate) -----------------------------------------------------------------
ESTIMATE_MODEL = [-1000.0, 1000.0, 0.0, 0.0, 160.0, 1000.0, 1000.0, 0.0, 0.0, 160.0]
BENCH_ASTIG = [150.0, 400.0, 0.05, 0.0, 1.3 * 160, -150.0, 400.0, -0.05, 0.0, 1.3 * 160]


def _astig_widths(model, z, pixel_size=160.0):
    out = []
    for k in (0, 5):
        z0, w, c3, c4, a = model[k:k + 5]
        u = (z - z0) / w
        out.append(a / pixel_size * np.sqrt(np.maximum(0.0, 1 + u * u + c3 * u ** 3 + c4 * u ** 4)))
    return np.stack(out, axis=1)


def test_astig_estimation_matches_reference_bitwise(orc, ref):
    """The restated z estimate equals the reference build bit for bit (grid, Brent steps, score)."""
    rng = np.random.default_rng(11)
    for model, zmax in ((BENCH_ASTIG, 600.0), (ESTIMATE_MODEL, 500.0), ([-60.0, 300.0, 0.06, 0.02, 140.0, 60.0, 300.0, -0.06, 0.02, 140.0], 600.0)):
        z = rng.uniform(-1.2 * zmax, 1.2 * zmax, 3000)
        s = _astig_widths(model, z) * rng.normal(1.0, 0.05, (z.size, 2))
        s[:5] = [[0.0, 1.0], [-1.0, 2.0], [np.nan, 1.0], [1.0, np.inf], [1e-9, 1e-9]]  # degenerate widths
        a = orc.astig_estimation(s, 160.0, model, zmax)
        b = ref.astig_estimation(s, 160.0, model, zmax)
        assert np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("observed, expected", [(-600.0, -500.0), (-500.0, -500.0), (-499.0, -499.0), (-123.4, -123.4),
                                                (0.0, 0.0), (123.4, 123.4), (499.0, 499.0), (500.0, 500.0), (600.0, 500.0)])
def test_astig_estimation_reference_cases(orc, observed, expected):
    """The reference test's estimate cases (Tests_CPU/test_fit_AstigFit.cpp:37-50, 241-256): exact at the bounds,
    within 1 nm inside."""
    s = _astig_widths(ESTIMATE_MODEL, np.array([observed]))
    z, score = orc.astig_estimation(s, 160.0, ESTIMATE_MODEL, 500.0)[0]
    if abs(expected) == 500.0:
        assert z == expected
    else:
        assert abs(z - expected) <= 1.0 and -500.0 < z < 500.0
        assert score > 0.999


def test_astig_estimation_recovers_noisy_z(orc):
    """Reference test Estimate (test_fit_AstigFit.cpp:223-238): 0.02 px noise, z in [-200, 200], within 40 nm, score
    > 0.95."""
    model = [-60.0, 300.0, 0.06, 0.02, 140.0, 60.0, 300.0, -0.06, 0.02, 140.0]
    rng = np.random.default_rng(42)
    z = rng.uniform(-200.0, 200.0, 10)
    s = _astig_widths(model, z) + rng.normal(0.0, 0.02, (10, 2))
    r = orc.astig_estimation(s, 160.0, model, 800.0)
    assert np.all(np.abs(r[:, 0] - z) <= 40.0) and np.all(r[:, 1] > 0.95) and np.all(r[:, 1] <= 1.0)


def test_bench_reference_arm_threshold(orc):
    # bench.py's reference arm takes the threshold from the reference build's own Wavelett (the oracle port without
    # it): it must be the MAD threshold of the frame's W1 plane, the value the GPU arm computes from its bit-exact plane
    import os
    import sys
    import synth
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import bench
    s, _ = synth.stack("c2", frames=1, seed=3, size=(256, 256))
    assert bench.reference_threshold(s[0]) == synth.mad_threshold(orc.planes(s[0])[1])
