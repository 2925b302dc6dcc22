"""Level pipeline on the GPU: residual target bit-identical to the torch
expression of train.py:113-126, the fused compose against F.interpolate +
the de-normalisation of train.py:193-200, and a checkpoint decode."""
import pytest
import torch
import torch.nn.functional as F

from lig_b200 import gsplat2d, synthetic
from lig_b200.levels import compose, decode_lig, load_lig, residual_target, save_lig
from lig_b200.serve import GaussianSet

pytestmark = pytest.mark.gpu


def test_residual_target_bit_identical_to_torch():
    g = torch.Generator().manual_seed(21)
    gt = torch.rand(333, 517, 3, generator=g).cuda()
    up = (torch.rand(333, 517, 3, generator=g) * 1.2 - 0.1).cuda()
    t, lo, hi = residual_target(gt, up)
    r = gt - up + 0.5
    elo, ehi = r.min(), r.max()
    assert torch.equal(lo, elo) and torch.equal(hi, ehi)
    assert torch.equal(t, (r - elo) / (ehi - elo))


@pytest.mark.parametrize("prev_hw,hw", [((50, 70), (100, 140)), ((64, 64), (250, 130)),
                                        ((90, 90), (90, 90)), ((120, 80), (61, 47))])
def test_compose_matches_interpolate(prev_hw, hw):
    g = torch.Generator().manual_seed(22)
    prev = (torch.rand(*prev_hw, 3, generator=g) * 1.4 - 0.2).cuda()
    render = (torch.rand(*hw, 3, generator=g) * 1.4 - 0.2).cuda()
    lo, hi = -0.3125, 1.1875
    for last in (False, True):
        out = compose(prev, render, lo, hi, last)
        up = F.interpolate(prev.permute(2, 0, 1).unsqueeze(0), size=hw, mode="bilinear")
        up = up.squeeze(0).permute(1, 2, 0)
        exp = up + (torch.clamp(render, 0, 1) * (hi - lo) - 0.5 + lo)
        if last:
            exp = torch.clamp(exp, 0, 1)
        # a few float ulps at |values| <= 2.5: bilinear weights may contract
        # into FMAs differently from torch's build
        assert (out - exp).abs().max().item() <= 4e-6
    # device min/max operands give the same result as host floats
    out_t = compose(prev, render, torch.tensor(lo).cuda(), torch.tensor(hi).cuda(), True)
    assert torch.equal(out_t, compose(prev, render, lo, hi, True))


def test_checkpoint_decode_matches_reference_decode(tmp_path):
    H, W = 96, 128
    lv = []
    for s, (h, w, n) in enumerate([(48, 64, 600), (96, 128, 1500)]):
        mu, ch, co = synthetic.gaussians(n, h, w, diag=(0.5, 3.0), seed=40 + s)
        lv.append(GaussianSet(mu.cuda(), ch.cuda(), co.cuda(), h, w))
    p = tmp_path / "m.pth.tar"
    save_lig(p, lv, [-0.2], [1.3])
    m = load_lig(p)
    out = decode_lig(m)
    # train.py:181-200 with the gsplat2d API: clamped level renders, bilinear
    # resize of the running image, de-normalised residual, final clamp
    renders = []
    for gs in lv:
        x, e, c, k = gsplat2d.project_gaussians_cholesky(gs.chol, gs.means, gs.H, gs.W, 16)
        renders.append(torch.clamp(gsplat2d.rasterize_gaussians(x, e, c, k, gs.rgbs, None, gs.H,
                                                                gs.W, 16)[0], 0, 1))
    est = renders[1] * (1.3 - (-0.2)) - 0.5 + (-0.2)
    up = F.interpolate(renders[0].permute(2, 0, 1).unsqueeze(0), size=(H, W), mode="bilinear")
    exp = torch.clamp(up.squeeze(0).permute(1, 2, 0) + est, 0, 1)
    assert (out - exp).abs().max().item() <= 2e-6
