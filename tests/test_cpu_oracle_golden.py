"""Pin the oracle: the C restatement against golden vectors produced by the
reference itself — its CUDA kernels (tests/golden/ref_*.npz, made by
tests/golden/make_golden_ref.py on a GPU from oracle/_ref) and its pure-torch
upscaler (tests/golden/torch_upscaler.npz, made by make_golden_torch.py).

Integer outputs must match exactly.  Float outputs differ only by rounding:
the reference runs --use_fast_math (__expf, approximate log/sqrt/division,
FMA contraction) while the oracle is plain IEEE, so images match to 1e-5 and
tile counts match except where the SnugBox value sits within rounding of an
integer (checked in FP64)."""
import glob
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.environ.get("LIG_GOLDEN_DIR",
                        os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
REF_CASES = sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


def _load(path):
    return dict(np.load(path))


def _near_integer_boundary(d, i):
    """True if Gaussian i's SnugBox extent or bbox edge is within float
    rounding of an integer (fast-math vs IEEE can then round differently)."""
    l11, l21, l22 = (float(v) for v in d["chol"][i])
    a, b, c = l11 * l11, l11 * l21, l21 * l21 + l22 * l22
    o = float(d["opac"][i]) if "opac" in d else 1.0
    t = 2 * math.log(255 * o)
    B = int(d["B"])
    x, y = (float(v) for v in d["means"][i])
    vals = []
    if t > 0:
        ex, ey = math.sqrt(t * a), math.sqrt(t * c)
        vals += [ex, ey]
        ex, ey = math.ceil(ex), math.ceil(ey)
        vals += [(x - ex) / B, (x + ex) / B + 1, (y - ey) / B, (y + ey) / B + 1]
    else:
        vals += [t]
    return any(abs(v - round(v)) < 1e-4 * max(1.0, abs(v)) for v in vals)


@pytest.mark.parametrize("path", REF_CASES, ids=[os.path.basename(p) for p in REF_CASES])
def test_oracle_projection_and_binning_vs_reference_kernels(path):
    d = _load(path)
    H, W, B = int(d["H"]), int(d["W"]), int(d["B"])
    op = d.get("opac")
    xys, ext, con, cnt = O.project_fwd(d["chol"], d["means"], op, H, W, B, chol=True)
    diff = np.nonzero(cnt != d["counts"])[0]
    assert all(_near_integer_boundary(d, i) for i in diff), diff
    ok = np.ones(len(cnt), bool)
    ok[diff] = False
    assert np.array_equal(ext[ok], d["extents"][ok])
    assert np.abs(con - d["conics"]).max() <= 2e-6 * max(1.0, np.abs(d["conics"]).max())
    # binning from the reference's own projection outputs: exact
    bn = O.bin_and_sort(d["xys"], d["extents"], d["counts"], H, W, B)
    assert np.array_equal(bn.cum_tiles_hit, d["cum"])
    assert np.array_equal(bn.isect_ids, d["isect_ids"])
    assert np.array_equal(bn.gaussian_ids, d["gids"])
    assert np.array_equal(bn.isect_ids_sorted, d["isect_sorted"])
    assert np.array_equal(bn.gaussian_ids_sorted, d["gid_sorted"])
    assert np.array_equal(bn.tile_bins, d["tile_bins"])


@pytest.mark.parametrize("path", REF_CASES, ids=[os.path.basename(p) for p in REF_CASES])
@pytest.mark.parametrize("tag", ["sum", "ga"])
def test_oracle_raster_vs_reference_kernels(path, tag):
    d = _load(path)
    H, W, B = int(d["H"]), int(d["W"]), int(d["B"])
    op = d.get("opac")
    ga = tag == "ga"
    bn = O.bin_and_sort(d["xys"], d["extents"], d["counts"], H, W, B)
    r = O.raster_fwd(H, W, B, bn, d["xys"], d["conics"], d["colors"], op, grad_aware=ga)
    # alpha-threshold flips (expf vs __expf) may move single pixels by <= 1/255 * colour
    bad = np.abs(r["img"] - d[f"{tag}_img"]).max(axis=-1) > 1e-5
    assert bad.mean() <= 1e-3
    assert np.abs(r["img"] - d[f"{tag}_img"]).max() <= 1.0 / 255 + 1e-5
    assert (r["final_idx"] != d[f"{tag}_final_idx"]).mean() <= 1e-3
    if ga:
        for k in ("dx", "dy", "dxy"):
            close = np.abs(r[k] - d[f"ga_{k}"]).max(axis=-1) <= 1e-4
            assert close.mean() >= 0.999, k
    vd = [d["v_dx"], d["v_dy"], d["v_dxy"]] if ga else [None] * 3
    g = O.raster_bwd(H, W, B, bn, d["xys"], d["conics"], d["colors"], op,
                     d[f"{tag}_final_idx"], d["v_img"], d["v_wsum"], *vd)
    for k in ("v_xy", "v_xy_abs", "v_conic", "v_rgb", "v_opacity"):
        key = f"{tag}_{k}"
        if key not in d:
            assert g[k] is None
            continue
        err = np.abs(g[k] - d[key]).max() / (np.abs(d[key]).max() + 1e-30)
        assert err <= 1e-4, (k, err)


@pytest.mark.parametrize("path", REF_CASES, ids=[os.path.basename(p) for p in REF_CASES])
def test_oracle_projection_backward_and_upscale_vs_reference_kernels(path):
    d = _load(path)
    v_chol, v_mean = O.project_bwd(d["extents"], d["chol"], d["conics"], d["pb_v_xy"],
                                   d["pb_v_conic"], chol=True)
    assert np.array_equal(v_mean, d["pb_v_mean"])
    err = np.abs(v_chol - d["pb_v_chol"]).max() / np.abs(d["pb_v_chol"]).max()
    assert err <= 1e-5
    planes = [d["up_f"], d["up_fx"], d["up_fy"], d["up_fxy"]]
    for tag, roi in (("full", None), ("roi", tuple(float(v) for v in d["up_roi"]))):
        dh, dw = d[f"up_{tag}_out"].shape[:2]
        sh, sw = planes[0].shape[:2]
        # the reference divides with fast-math approximate division: the source
        # coordinate (up to ~sw) moves by ~1 ulp, the spline by ~|slope| * ulp
        tol = 1e-4
        out = O.upscale_fwd(*planes, dh, dw, roi=roi, mode=0)
        assert np.abs(out - d[f"up_{tag}_out"]).max() <= tol * max(1, np.abs(out).max())
        gs = O.upscale_bwd(d[f"up_{tag}_g"], sh, sw, roi=roi, mode=0)
        for k, gg in zip(("gf", "gfx", "gfy", "gfxy"), gs):
            ref = d[f"up_{tag}_{k}"]
            assert np.abs(gg - ref).max() <= tol * max(1.0, np.abs(ref).max()), k


def test_oracle_align_corners_upscale_vs_reference_torch():
    d = _load(os.path.join(GOLDEN, "torch_upscaler.npz"))
    for t in "abc":
        h, w, nh, nw = (int(v) for v in d[f"{t}_shape"])
        out = O.upscale_fwd(d[f"{t}_f"], d[f"{t}_fx"], d[f"{t}_fy"], d[f"{t}_fxy"], nh, nw,
                            mode=1)
        assert np.abs(out - d[f"{t}_out"]).max() <= 1e-5 * max(1.0, np.abs(out).max())
        for k, g in zip(("gf", "gfx", "gfy", "gfxy"), O.upscale_bwd(d[f"{t}_go"], h, w, mode=1)):
            ref = d[f"{t}_{k}"]
            assert np.abs(g - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max()), k


def test_golden_fixtures_present():
    assert REF_CASES, "reference-kernel golden vectors missing (tests/golden/ref_*.npz)"
