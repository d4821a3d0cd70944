"""The CPU oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py). Runs without a GPU."""
import numpy as np
import pytest

from conftest import golden, rel_l2
from oracle import bp as obp
from oracle import filter as of
from oracle import geometry as og
from oracle import phantom as oph
from oracle.recon import OracleReconstructor


class _Geo:
    def __init__(self, **kw):
        self.box = None
        self.__dict__.update(kw)


def test_ramp_response_matches_reference():
    g = golden("ramp.npz")
    for key, H in g.items():
        _, n, tau, w = key.split("_", 3)
        Ho, N = of.ramp_response(int(n), float(tau), w)
        assert N == len(H)
        np.testing.assert_allclose(Ho, H, rtol=0, atol=1e-12 * np.abs(H).max())


def test_ramp_response_rejects_unknown_window():
    with pytest.raises(ValueError):
        of.ramp_response(16, 1.0, "gaussian")


def test_filter_rows_matches_reference():
    g = golden("filter_rows.npz")
    for w in ("ram-lak", "shepp-logan", "hann", "cosine"):
        y = of.filter_rows(g["x"], 0.9, w)
        assert y.dtype == np.float32
        np.testing.assert_array_equal(y, g[f"y_{w}"])
    y64 = of.filter_rows(g["x"].astype(np.float64), 0.9, "shepp-logan")
    np.testing.assert_allclose(y64, g["y64_shepp-logan"], rtol=0, atol=1e-6)


def test_cone_constants_and_fdk_block_match_reference():
    g = golden("fdk.npz")
    K = of.cone_constants(g["V_gen"])
    for k in K:
        np.testing.assert_allclose(K[k], g["K_" + k], rtol=1e-14, atol=1e-12)
    for w in ("shepp-logan", "ram-lak"):
        out = of.fdk_filter_block(g["block"], K, w)
        np.testing.assert_allclose(out, g[f"fdk_{w}"], rtol=0, atol=1e-6 * np.abs(g[f"fdk_{w}"]).max())
    par = of.parallel_filter_block(g["block"], 0.8, "hann")
    np.testing.assert_array_equal(par, g["par_hann"])


def test_c_backprojection_matches_numba():
    g = golden("bp.npz")
    K = of.cone_constants(g["V"])
    D = K["d"] - float(g["shift"]) * K["u"]
    A = g["q"].shape[0]
    out = obp.bp_cone(g["q"], K["s"], D, K["uu"], K["vv"], K["n"], K["sdd"], K["sod"], g["pts"], np.pi / A)
    np.testing.assert_allclose(out, g["cone_numba"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(out, g["cone_numpy"], rtol=1e-9, atol=1e-12)
    a = g["angles"]
    out = obp.bp_parallel(g["q"], np.cos(a), np.sin(a), 0.9, 1.1, g["pts"], np.pi / A, -1.3)
    np.testing.assert_allclose(out, g["par_numba"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(out, g["par_numpy"], rtol=1e-9, atol=1e-12)


def test_c_backprojection_threads_do_not_change_results():
    g = golden("bp.npz")
    K = of.cone_constants(g["V"])
    pts = np.repeat(g["pts"], 8, axis=0)      # > 1024 points: the threaded path
    args = (g["q"], K["s"], K["d"], K["uu"], K["vv"], K["n"], K["sdd"], K["sod"], pts, 0.5)
    old = obp.threads(0)
    obp.threads(1)
    one = obp.bp_cone(*args)
    obp.threads(4)
    four = obp.bp_cone(*args)
    obp.threads(old)
    np.testing.assert_array_equal(one, four)


def test_preprocess_matches_reference():
    g = golden("preprocess.npz")
    np.testing.assert_allclose(of.gaussian_blur(g["block"], 1.5), g["gauss_1_5"], atol=1e-6)
    np.testing.assert_array_equal(of.rotate_projections(g["block"], 7.0), g["rot_7"])
    np.testing.assert_allclose(of.preprocess_apply(g["block"], 0.8, 2.5), g["apply"], atol=1e-6)
    rot = of.rotate_projections(g["point"], 90.0)
    np.testing.assert_array_equal(rot, g["rot_90"])


def test_phantom_matches_reference():
    g = golden("phantom.npz")
    ph = oph.Phantom(scale=50.0)
    np.testing.assert_array_equal(ph.evaluate(g["pts"]), g["evaluate"])
    np.testing.assert_allclose(ph.line_integrals(g["starts"], g["dirs"]), g["lines"], rtol=1e-12, atol=1e-12)
    par = oph.project_parallel(ph, np.arange(9) * np.pi / 9, 10, 12, 9.0, 11.0)
    np.testing.assert_allclose(par, g["par"], rtol=1e-6, atol=1e-5)
    V = og.circular_cone_vectors(9, 300.0, 600.0, 15.0, det_shift_u=1.5)
    np.testing.assert_allclose(V, g["cone_V"], rtol=1e-15, atol=1e-12)
    np.testing.assert_allclose(oph.project_cone(ph, V, 10, 12), g["cone"], rtol=1e-6, atol=1e-5)


@pytest.mark.parametrize("name", ["cone", "parallel"])
def test_oracle_reconstructor_matches_reference(name):
    g = golden(f"recon_{name}.npz")
    if name == "cone":
        geo = _Geo(vectors=g["V"], rows=int(g["rows"]), cols=int(g["cols"]))
    else:
        geo = _Geo(angles=g["angles"], rows=int(g["rows"]), cols=int(g["cols"]), pixel_u=3.5, pixel_v=4.4)
    rec = OracleReconstructor(g["proj"], geo)
    np.testing.assert_allclose(rec.box, g["box"], rtol=1e-15)
    tol = 1e-6 * np.abs(g["img_oblique"]).max()
    img, _ = rec.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=40, size=110)
    np.testing.assert_allclose(img, g["img_oblique"], rtol=0, atol=tol)
    img, _ = rec.reconstruct_plane((0, 0, 1.0), (0.3, 0.0, 1.0), n=33, zoom=1.5, center=(2.0, 0, 0),
                                   cor_shift=0.8)
    np.testing.assert_allclose(img, g["img_zoom"], rtol=0, atol=tol)
    img, _ = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=24)
    np.testing.assert_allclose(img, g["img_axial"], rtol=0, atol=tol)
    vol, origin, h = rec.reconstruct_volume(voxel=8.0)
    np.testing.assert_allclose(origin, g["vol_origin"])
    assert h == float(g["vol_h"])
    np.testing.assert_allclose(vol, g["vol"], rtol=0, atol=tol)
    best, scores = rec.estimate_cor(np.arange(-2.0, 2.01, 0.5), n=32)
    np.testing.assert_allclose(scores, g["cor_scores"], rtol=1e-9)
    assert best == float(g["cor_best"])
    # streaming in interleaved order == the reference's live reconstruction
    live = OracleReconstructor(None, geo)
    order = og.arrival_order(live.n_total, "interleaved")
    for i in range(0, len(order), 7):
        live.add_projections(order[i:i + 7], g["proj"][:, order[i:i + 7], :])
    np.testing.assert_array_equal(live._order[:live.n], g["live_order"])
    img, _ = live.reconstruct_plane((0, 0, 1.0), (0.3, 0.0, 1.0), n=33, zoom=1.5, center=(2.0, 0, 0),
                                    cor_shift=0.8)
    np.testing.assert_allclose(img, g["img_live"], rtol=0, atol=tol)


def test_fp64_oracle_is_close_to_reference_numerics():
    g = golden("recon_cone.npz")
    geo = _Geo(vectors=g["V"], rows=int(g["rows"]), cols=int(g["cols"]))
    r64 = OracleReconstructor(g["proj"], geo, precision="fp64")
    img, _ = r64.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=40, size=110)
    assert rel_l2(img, g["img_oblique"]) < 1e-6


def test_raw_correction_matches_reference_loaders():
    g = golden("loaders.npz")
    proj, _, _ = of.hdf5_correct(g["h5_data"], g["h5_white"], g["h5_dark"], 2)
    np.testing.assert_allclose(np.transpose(proj, (1, 0, 2)), g["h5_proj"], rtol=1e-6, atol=1e-6)
    fx, _, _ = of.flexray_correct(g["fx_raw"], g["fx_dark"], g["fx_flat"], 2)
    np.testing.assert_allclose(np.transpose(fx, (1, 0, 2)), g["fx_proj"], rtol=1e-6, atol=1e-6)


def test_arrival_order_matches_reference():
    g = golden("misc.npz")
    for n in (1, 2, 10, 17, 64, 600):
        np.testing.assert_array_equal(og.arrival_order(n, "interleaved"), g[f"order_{n}"])
