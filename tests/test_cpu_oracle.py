"""CPU checks of the oracle (the C restatement) itself: FP64 tile path equals
the FP64 dense evaluator, backward equals FP64 finite differences, binning
invariants, reference edge cases (empty list, zero-extent slots), and the
upscale forward/backward adjoint identity."""
import numpy as np
import pytest

from oracle import oracle as O

F64 = np.float64


def _scene(n, H, W, diag=(0.5, 4.0), seed=0, opac=None):
    rng = np.random.default_rng(seed)
    means = np.stack([rng.uniform(0, W, n), rng.uniform(0, H, n)], 1)
    chol = np.stack([rng.uniform(*diag, n), rng.normal(0, 0.5, n), rng.uniform(*diag, n)], 1)
    cols = rng.uniform(0, 1, (n, 3))
    op = None if opac is None else rng.uniform(*opac, n)
    return means, chol, cols, op


@pytest.mark.parametrize("B", [16, 8, 12, 5])
@pytest.mark.parametrize("ga", [False, True])
def test_tile_path_equals_dense_fp64(B, ga):
    H, W = 61, 77
    means, chol, cols, op = _scene(250, H, W, opac=(0.05, 1.0), seed=B)
    r = O.render(chol, means, cols, op, H, W, B, chol=True, grad_aware=ga, dtype=F64)
    d = O.dense_fwd_f64(H, W, B, r["xys"], r["extents"], r["counts"], r["conics"], cols, op,
                        grad_aware=ga)
    for k in ("img", "wsum") + (("dx", "dy", "dxy") if ga else ()):
        assert np.abs(d[k] - r[k]).max() <= 1e-12, k


def test_zero_extent_slots_land_in_tile_zero():
    """Opacity < 1/255 gives extent 0 but a tile count of 1 (reference
    csrc/forward.cu:84-88 + :44-52); map_gaussian_to_intersects leaves those
    slots as key 0 / id 0 (csrc/forward.cu:123-124)."""
    H, W, B = 64, 64, 16
    means = np.array([[40.0, 40.0], [10.0, 50.0], [20.0, 20.0]])
    chol = np.array([[2.0, 0.0, 2.0], [2.0, 0.3, 1.0], [1.5, 0.0, 1.5]])
    op = np.array([0.9, 0.002, 0.8])
    xys, ext, con, cnt = O.project_fwd(chol, means, op, H, W, B, chol=True, dtype=F64)
    assert cnt[1] == 1 and ext[1, 0] == 0 and ext[1, 1] == 0
    bn = O.bin_and_sort(xys, ext, cnt, H, W, B, dtype=F64)
    start = bn.cum_tiles_hit[0]
    assert bn.isect_ids[start] == 0 and bn.gaussian_ids[start] == 0
    t0 = bn.tile_bins[0]
    assert 0 in bn.gaussian_ids_sorted[t0[0]:t0[1]]
    d = O.dense_fwd_f64(H, W, B, xys, ext, cnt, con, np.ones((3, 3)), op)
    r = O.raster_fwd(H, W, B, bn, xys, con, np.ones((3, 3)), op, dtype=F64)
    assert np.abs(d["img"] - r["img"]).max() <= 1e-12


def test_empty_intersections_give_white_image():
    H, W, B = 32, 40, 16
    means = np.array([[-100.0, -100.0]])
    chol = np.array([[1.0, 0.0, 1.0]])
    r = O.render(chol, means, np.ones((1, 3)), None, H, W, B, chol=True, grad_aware=True)
    assert r["binning"].num_intersects == 0
    assert np.all(r["img"] == 1) and np.all(r["wsum"] == 0) and np.all(r["dx"] == 0)


def test_binning_invariants():
    H, W, B = 96, 128, 16
    means, chol, cols, op = _scene(600, H, W, diag=(0.5, 6.0))
    xys, ext, con, cnt = O.project_fwd(chol, means, op, H, W, B, chol=True)
    bn = O.bin_and_sort(xys, ext, cnt, H, W, B)
    tiles = bn.isect_ids_sorted >> 32
    assert np.all(np.diff(tiles) >= 0)
    for t in range(bn.tile_bins.shape[0]):
        a, b = bn.tile_bins[t]
        if a == b:
            assert a == 0 and b == 0
            continue
        assert np.all(tiles[a:b] == t)
        assert np.all(np.diff(bn.gaussian_ids_sorted[a:b]) > 0)  # stable: ascending id


def _fd_check(ga, clamp, names):
    H, W, B = 48, 40, 16
    means, chol, cols, op = _scene(60, H, W, diag=(1.0, 4.0), opac=(0.3, 0.9), seed=7)
    r = O.render(chol, means, cols, op, H, W, B, chol=True, grad_aware=ga, dtype=F64)
    bn, xys, con = r["binning"], r["xys"], r["conics"]
    rng = np.random.default_rng(1)
    ws = [rng.normal(size=s) for s in [(H, W, 3), (H, W), (H, W, 3), (H, W, 3), (H, W, 3)]]
    keys = ["img", "wsum", "dx", "dy", "dxy"] if ga else ["img", "wsum"]

    def loss(xys, con, cols, op):
        o = O.raster_fwd(H, W, B, bn, xys, con, cols, op, grad_aware=ga, dtype=F64)
        return sum((o[k] * w).sum() for k, w in zip(keys, ws))

    vd = ws[2:] if ga else [None] * 3
    g = O.raster_bwd(H, W, B, bn, xys, con, cols, op, r["final_idx"], ws[0], ws[1], *vd,
                     clamp=clamp, dtype=F64)
    h = 1e-6
    args = dict(xys=xys, con=con, cols=cols, op=op)
    gk = dict(xys="v_xy", con="v_conic", cols="v_rgb", op="v_opacity")
    for name in names:
        arr = args[name]
        for _ in range(10):
            idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
            vals = []
            for dlt in (h, -h, 2 * h, -2 * h):
                a = dict(args)
                a[name] = arr.copy()
                a[name][idx] += dlt
                vals.append(loss(**a))
            fd1 = (vals[0] - vals[1]) / (2 * h)
            fd2 = (vals[2] - vals[3]) / (4 * h)
            if abs(fd1 - fd2) > 1e-4 * (abs(fd1) + 1e-3):
                continue  # culling threshold crossed
            an = g[gk[name]][idx]
            assert abs(an - fd1) <= 1e-5 * (abs(fd1) + 1e-2), (name, idx, an, fd1)


def test_sum_backward_matches_fd():
    # clamp 0.999: the exact derivative of the 0.999-clamped forward
    _fd_check(False, 0.999, ["xys", "con", "cols", "op"])


def test_gradient_aware_backward_matches_fd():
    # the reference's opacity gradient in this kernel omits the dx/dy/dxy paths
    # (csrc/gradient_aware_rasterizer.cu:313-314), so opacity is not FD-exact
    _fd_check(True, 0.999, ["xys", "con", "cols"])


@pytest.mark.parametrize("mode,roi", [(0, None), (0, (3.0, 2.0, 30.5, 22.0)), (1, None)])
def test_upscale_backward_is_adjoint(mode, roi):
    rng = np.random.default_rng(4)
    h, w, dh, dw = 24, 33, 61, 80
    planes = [rng.normal(size=(h, w, 3)) for _ in range(4)]
    g = rng.normal(size=(dh, dw, 3))
    out = O.upscale_fwd(*planes, dh, dw, roi=roi, mode=mode, dtype=F64)
    grads = O.upscale_bwd(g, h, w, roi=roi, mode=mode, dtype=F64)
    lhs = (out * g).sum()
    rhs = sum((p * q).sum() for p, q in zip(planes, grads))
    assert abs(lhs - rhs) <= 1e-10 * (abs(lhs) + 1)


def test_upscale_identity_at_same_size():
    rng = np.random.default_rng(5)
    h, w = 20, 27
    planes = [rng.normal(size=(h, w, 3)) for _ in range(4)]
    out = O.upscale_fwd(*planes, h, w, mode=1, dtype=F64)  # align corners: exact grid points
    assert np.abs(out - planes[0]).max() <= 1e-12
