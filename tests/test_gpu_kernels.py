"""GPU parity of each drop-in kernel against the reference's golden vectors
(tests/golden/kernels.npz), called through the C ABI via the mirror modules.

Bit-exact expectations: interpolation (linear and nearest-row branches),
Laplacian, fused divergence, gradients/fluxes, abs_max, clamp, update.
The elastic update goes through cuFFT instead of pocketfft, so it is held to
1e-12 relative (of the elastic term's scale) instead.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ELASTIC_RTOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_interpolation_bitwise(torch_cuda, small_table, kernels_golden):
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    g = kernels_golden
    pts = g["interp_points"]
    out = np.empty((pts.shape[0], 9))
    mask = np.empty(pts.shape[0], dtype=np.bool_)
    interpolator_nb(pts, small_table["grid"], small_table["resolution"], small_table["tree"],
                    small_table["vals"], out=out, mask_buffer=mask)
    assert np.array_equal(mask, g["interp_mask"])
    assert np.array_equal(out, g["interp_out"])


def test_interpolation_torch_inplace(torch_cuda, small_table, kernels_golden):
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    t = torch_cuda
    g = kernels_golden
    pts = t.from_numpy(g["interp_points"]).cuda()
    grid = t.from_numpy(small_table["grid"]).cuda()
    out = t.empty((pts.shape[0], 9), dtype=t.float64, device="cuda")
    res = interpolator_nb(pts, grid, small_table["resolution"], small_table["tree"],
                          small_table["vals"], out=out)
    assert res.data_ptr() == out.data_ptr()
    assert np.array_equal(out.cpu().numpy(), g["interp_out"])


def test_interpolation_max_nn_dist_raises(torch_cuda, small_table):
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    far = np.array([[0.6, 0.6, 0.0, 0.0]])
    with pytest.raises(RuntimeError):
        interpolator_nb(far, small_table["grid"], small_table["resolution"], small_table["tree"],
                        small_table["vals"], max_nn_dist=1e-3)


def test_nearest_row_matches_kdtree_property(torch_cuda, small_table):
    """Random points beyond the linear threshold: device nearest node == cKDTree."""
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    rng = np.random.default_rng(5)
    x = rng.dirichlet(np.ones(5), size=4000)[:, 1:] * rng.uniform(0.85, 1.0, size=(4000, 1))
    out = np.empty((x.shape[0], 9))
    mask = np.empty(x.shape[0], dtype=np.bool_)
    interpolator_nb(x, small_table["grid"], small_table["resolution"], small_table["tree"],
                    small_table["vals"], out=out, mask_buffer=mask)
    bad = ~mask
    assert bad.sum() > 1000
    _, nn = small_table["tree"].query(x[bad])
    assert np.array_equal(out[bad], small_table["vals"][nn])


def _off_simplex_points(seed):
    """Points a window-limited search could miss: row sums in [1.05, 1.5],
    components far outside [0, 1], and a few hand-picked extremes."""
    rng = np.random.default_rng(seed)
    s = rng.uniform(1.05, 1.5, size=(3000, 1))
    beyond = rng.dirichlet(np.ones(4), size=3000) * s
    far = rng.uniform(-0.6, 1.6, size=(3000, 4))
    picked = np.array([[1.2, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 2.0], [5.0, 5.0, 5.0, 5.0],
                       [-3.0, 0.1, 0.1, 0.1], [0.6, 0.6, 0.0, 0.0], [1.0, 1.0, 1.0, 1.0],
                       [-1.0, -1.0, -1.0, -1.0], [0.3, 0.3, 0.3, 0.3], [40.0, -7.0, 0.2, 0.9]])
    return np.concatenate([beyond, far, picked])


def test_nearest_row_exact_off_simplex(torch_cuda, small_table):
    """Every point outside the linear region -- including points well past the
    simplex face and far outside [0, 1] -- gets exactly the row the
    reference's cKDTree returns, and the whole output (linear branch
    included) equals the oracle's bit for bit."""
    from oracle import oracle as O
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    x = _off_simplex_points(17)
    t = small_table
    out = np.empty((x.shape[0], 9))
    mask = np.empty(x.shape[0], dtype=np.bool_)
    interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"], out=out,
                    mask_buffer=mask)
    bad = ~mask
    assert bad.sum() > 4000
    _, nn = t["tree"].query(x[bad])
    assert np.array_equal(out[bad], t["vals"][nn])
    ref = O.interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"])
    assert np.array_equal(out, ref, equal_nan=True)


def test_nearest_row_exact_on_fine_table(torch_cuda):
    """The same property on the 0.025-spacing (41^4) workload table, whose
    windows are narrower in composition units."""
    from phasefield5d_b200 import workload as W
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    from phasefield5d_b200.solver.table import build_4d_grid, build_calphad_kdtree
    data = W.make_table(0.025, 873.0, 4).data
    _, grid = build_4d_grid(data, 0.025)
    tree, vals = build_calphad_kdtree(data)
    x = _off_simplex_points(23)
    out = np.empty((x.shape[0], 9))
    mask = np.empty(x.shape[0], dtype=np.bool_)
    interpolator_nb(x, grid, 0.025, tree, vals, out=out, mask_buffer=mask)
    bad = ~mask
    _, nn = tree.query(x[bad])
    assert np.array_equal(out[bad], vals[nn])


def test_nearest_row_nonfinite_raises(torch_cuda, small_table):
    """A NaN composition reaches the fallback (NaN <= threshold is false);
    the reference's cKDTree.query raises ValueError for it, and so does the
    device path."""
    from oracle import oracle as O
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    t = small_table
    x = np.array([[0.1, 0.2, 0.1, 0.1], [np.nan, 0.2, 0.1, 0.1]])
    with pytest.raises(ValueError):
        O.interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"])
    with pytest.raises(ValueError):
        interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"])


def test_nearest_row_far_off_simplex_distance_error(torch_cuda, small_table):
    """x = (1.2, 0, 0, 0) is 0.2 from its nearest row (1, 0, 0, 0): with
    max_nn_dist = 0.1 both the reference and the device raise."""
    from oracle import oracle as O
    from phasefield5d_b200.solver.interpolation import interpolator_nb
    t = small_table
    x = np.array([[1.2, 0.0, 0.0, 0.0]])
    with pytest.raises(RuntimeError):
        O.interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"], max_nn_dist=0.1)
    with pytest.raises(RuntimeError):
        interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"], max_nn_dist=0.1)
    out = interpolator_nb(x, t["grid"], t["resolution"], t["tree"], t["vals"], max_nn_dist=0.25)
    _, nn = t["tree"].query(x)
    assert np.array_equal(out, t["vals"][nn])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_laplacian_bitwise(torch_cuda, kernels_golden, dim):
    from phasefield5d_b200.solver.operators import calculate_laplacian
    g = kernels_golden
    out = calculate_laplacian(g[f"lap{dim}_X"], float(g["dx"]))
    assert np.array_equal(out, g[f"lap{dim}_out"])


def test_laplacian_two_components_zero_sum(torch_cuda):
    """Reference test_smoke.py:24-40 pattern (S = 2, periodic zero sum)."""
    from phasefield5d_b200.solver.operators import calculate_laplacian
    rng = np.random.default_rng(0)
    for shape in [(32, 2), (16, 16, 2)]:
        c = rng.random(shape)
        L = calculate_laplacian(c, 1.0)
        assert L.shape == c.shape
        np.testing.assert_allclose(L.sum(axis=tuple(range(c.ndim - 1))), 0.0, atol=1e-10)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_divergence_bitwise(torch_cuda, kernels_golden, dim):
    from phasefield5d_b200.solver.fluxes import get_divergence_from_mu_function
    g = kernels_golden
    X = g[f"lap{dim}_X"]
    buf = g[f"div{dim}_buf"]
    out = np.empty_like(X)
    get_divergence_from_mu_function(dim)(X, buf[..., 4:], buf[..., :4], 1.0 / float(g["dx"]), out)
    assert np.array_equal(out, g[f"div{dim}_out"])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_divergence_strided_views_bitwise(torch_cuda, kernels_golden, dim):
    """mu and M as strided views of one (…, 9) device buffer, as in the loop."""
    from phasefield5d_b200.solver.fluxes import get_divergence_from_mu_function
    t = torch_cuda
    g = kernels_golden
    X = t.from_numpy(g[f"lap{dim}_X"]).cuda()
    buf = t.from_numpy(g[f"div{dim}_buf"]).cuda()
    out = t.empty_like(X)
    get_divergence_from_mu_function(dim)(X, buf[..., 4:], buf[..., :4], 1.0 / float(g["dx"]), out)
    assert np.array_equal(out.cpu().numpy(), g[f"div{dim}_out"])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_gradients_and_fluxes_bitwise(torch_cuda, kernels_golden, dim):
    from phasefield5d_b200.solver.fluxes import get_flux_function
    from phasefield5d_b200.solver.operators import calculate_gradients_pm
    g = kernels_golden
    X = g[f"lap{dim}_X"]
    buf = g[f"div{dim}_buf"]
    gp, gm = calculate_gradients_pm(buf[..., :4], float(g["dx"]))
    assert np.array_equal(gp, g[f"grad{dim}_p"]) and np.array_equal(gm, g[f"grad{dim}_m"])
    fp = np.empty_like(gp)
    fm = np.empty_like(gm)
    get_flux_function(dim)(X, buf[..., 4:], gp, gm, fp, fm)
    assert np.array_equal(fp, g[f"flux{dim}_p"]) and np.array_equal(fm, g[f"flux{dim}_m"])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_elastic_update(torch_cuda, kernels_golden, dim):
    from phasefield5d_b200.solver.elastic import make_elastic_updater

    class Cfg:
        include_cubic_anisotropy = True
        initial_composition = kernels_golden["el_X0"]

    g = kernels_golden
    X = g[f"el{dim}_X"]
    lv = g[f"el{dim}_lvec"]
    lam = np.outer(lv, lv)
    mu = g[f"el{dim}_mu_in"].copy()
    upd = make_elastic_updater(Cfg(), lam, g[f"el{dim}_bk"], X.shape, np.float64)
    upd(mu, X)
    want = g[f"el{dim}_mu_out"]
    delta_ref = want - g[f"el{dim}_mu_in"]
    delta = mu - g[f"el{dim}_mu_in"]
    scale = np.max(np.abs(delta_ref))
    assert scale > 0
    # l enters twice, so the factor's arbitrary sign cancels
    assert np.max(np.abs(delta - delta_ref)) <= ELASTIC_RTOL * scale


def test_abs_max_clamp_update(torch_cuda, kernels_golden):
    from phasefield5d_b200.solver.operators import abs_max, clamp_simplex
    g = kernels_golden
    assert abs_max(g["absmax_in"]) == float(g["absmax_out"])
    X = g["clamp_in"].copy()
    clamp_simplex(X)
    assert np.array_equal(X, g["clamp_out"])
    assert abs_max(np.zeros(0)) == 0.0


def test_update_two_roundings(torch_cuda):
    from phasefield5d_b200 import _lib
    t = torch_cuda
    rng = np.random.default_rng(3)
    X = rng.random((1000, 4))
    dX = rng.normal(size=(1000, 4)) * 1e3
    dt = 2.576e-12
    Xd, dXd = t.from_numpy(X).cuda(), t.from_numpy(dX).cuda()
    _lib.check(_lib.load().pf5d_update(_lib.ptr(Xd), _lib.ptr(dXd), X.size, dt,
                                       _lib.stream_handle()))
    d = dX * dt
    assert np.array_equal(dXd.cpu().numpy(), d)
    assert np.array_equal(Xd.cpu().numpy(), X + d)


def test_out_of_bounds_matches_reference(torch_cuda, kernels_golden):
    from phasefield5d_b200.solver.operators import out_of_bounds
    g = kernels_golden
    for x, want in zip(g["oob_in"], g["oob_out"]):
        assert out_of_bounds(x) == bool(want)


def test_unsupported_dim_raises(torch_cuda):
    from phasefield5d_b200.solver.fluxes import get_divergence_from_mu_function
    from phasefield5d_b200.solver.operators import calculate_laplacian
    with pytest.raises(ValueError):
        get_divergence_from_mu_function(4)
    with pytest.raises(NotImplementedError):
        calculate_laplacian(np.zeros((2, 2, 2, 2, 4)), 1.0)
