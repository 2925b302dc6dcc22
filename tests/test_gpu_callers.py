"""LIG's own training code, unmodified, on this library vs on the reference.

Each test runs the reference's gaussianlig.py, train.py or
minimal_trainer_upscale.py (bytecode of the unmodified files; see
tests/_callers.py) twice in this process: once with `gsplat2d` /
`upscaler_torch` resolving to this library through
lig_b200.install_gsplat2d(), once with them resolving to the reference's own
gsplat2d package on the reference's kernels.  Same seeds, same target; the
comparison is on what LIG's code computes: renders (1e-5), gradients
(1e-4 relative), parameter updates (1e-4 relative) and PSNR (0.05 dB).

  * Gaussian2D.train_iter (gaussianlig.py:70-111): cov2d parameterisation,
    rgbs initialised to zeros, torch Adam at train.py's default lr 0.018.
  * SimpleTrainer2d.train (train.py:17-207): the two-level LIG loop with
    train.py's defaults (n_scales 2, allo_ratio 0.5, lr 0.018), including
    the residual / min-max level hand-over, the eval renders, checkpoint
    save and test(); a fit that learns (PSNR rises well above the start and
    level 2 improves on level 1).
  * Gaussian2DMinimal.forward + upscale_fn (minimal_trainer_upscale.py:
    75-170): Cholesky + opacity parameterisation, gradient-aware render,
    CUDA and torch upscalers, scale_to, and the reference's Adan (unfused).
"""
import argparse
import math

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import _callers
from _scene import rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _callers.available(),
                                 reason="reference caller bytecode / kernels not built "
                                        "(make -C oracle ref)")]

DEV = torch.device("cuda:0")


def _target(H, W, seed=5):
    """Smooth seeded RGB image in [0, 1], [1, 3, H, W] (NCHW, as train.py loads it)."""
    g = torch.Generator().manual_seed(seed)
    low = torch.rand(1, 3, max(H // 16, 2), max(W // 16, 2), generator=g)
    img = F.interpolate(low, size=(H, W), mode="bicubic", align_corners=False)
    img = img + 0.05 * torch.rand(1, 3, H, W, generator=g)
    return img.clamp(0, 1).to(DEV)


def _psnr(a, b):
    return 10 * math.log10(1.0 / F.mse_loss(a.float(), b.float()).item())


# ----------------------------------------------------------------- gaussianlig.py

def _gaussianlig_run(arm, gt, n, iters):
    H, W = gt.shape[2], gt.shape[3]
    with _callers.bound(arm):
        import gaussianlig
        torch.manual_seed(0)
        m = gaussianlig.Gaussian2D(loss_type="L2", opt_type="adam", num_points=n, H=H, W=W,
                                   BLOCK_H=16, BLOCK_W=16, device=DEV, lr=0.018)
        params = (m.means, m.cov2d, m.rgbs)
        init = [p.detach().clone() for p in params]
        grads, losses, psnrs = [], [], []
        step = m.optimizer.step

        def recording_step(*a, **k):
            grads.append([p.grad.detach().clone() for p in params])
            return step(*a, **k)

        m.optimizer.step = recording_step
        for _ in range(iters):
            loss, psnr = m.train_iter(gt)
            losses.append(float(loss))
            psnrs.append(psnr)
        with torch.no_grad():
            render = m.forward()["render"].detach().clone()
        return dict(init=init, grads=grads, losses=losses, psnrs=psnrs, render=render,
                    delta=[p.detach() - i for p, i in zip(params, init)],
                    origin=_callers.module_origin("gsplat2d"))


def test_gaussianlig_train_iter_matches_reference():
    gt = _target(96, 128)
    mine = _gaussianlig_run("lig", gt, 3000, 10)
    ref = _gaussianlig_run("ref", gt, 3000, 10)
    assert "lig_b200" in mine["origin"] and "_ref" in ref["origin"]
    for a, b in zip(mine["init"], ref["init"]):
        assert torch.equal(a, b)
    for it, (ga, gb) in enumerate(zip(mine["grads"], ref["grads"])):
        for name, a, b in zip(("means", "cov2d", "rgbs"), ga, gb):
            assert rel_err(a.cpu(), b.cpu()) < 1e-4, (it, name)
    np.testing.assert_allclose(mine["losses"], ref["losses"], rtol=1e-5)
    np.testing.assert_allclose(mine["psnrs"], ref["psnrs"], atol=1e-4)
    assert (mine["render"] - ref["render"]).abs().max().item() < 1e-5
    for name, a, b in zip(("means", "cov2d", "rgbs"), mine["delta"], ref["delta"]):
        assert rel_err(a.cpu(), b.cpu()) < 1e-4, name
    assert mine["psnrs"][-1] > mine["psnrs"][0] + 1.0   # the fit learns


# ----------------------------------------------------------------------- train.py

def _train_py_run(arm, png, tmp, n, iters):
    with _callers.bound(arm):
        import train
        torch.manual_seed(1)
        args = argparse.Namespace(save_imgs=False, n_scales=2, allo_ratio=0.5, lr=0.018)
        tr = train.SimpleTrainer2d(image_path=png, log_path=str(tmp / arm), num_points=n,
                                   model_name="LIG", iterations=iters, model_path=None,
                                   args=args)
        psnr, _, _, _, _ = tr.train()
        gm = tr.gaussian_model
        with torch.no_grad():
            lvl1 = gm.level_models[0]().get("render").float()
            up1 = F.interpolate(lvl1, size=(tr.H, tr.W), mode="bilinear")
            p1 = _psnr(torch.clamp(up1, 0, 1), tr.gt_image)
            p0 = _psnr(torch.zeros_like(tr.gt_image), tr.gt_image)
        ckpt = torch.load(tmp / arm / png.stem / "gaussian_model.pth.tar", map_location="cpu")
        return dict(psnr=psnr, level1=p1, start=p0, ckpt=ckpt,
                    origin=_callers.module_origin("gsplat2d"))


def test_train_py_two_level_psnr_matches_reference(tmp_path):
    from PIL import Image
    gt = _target(256, 256, seed=6)
    arr = (gt[0].permute(1, 2, 0).cpu().numpy() * 255).round().astype(np.uint8)
    png = tmp_path / "synthetic_0001.png"
    Image.fromarray(arr).save(png)
    mine = _train_py_run("lig", png, tmp_path, 12000, 300)
    ref = _train_py_run("ref", png, tmp_path, 12000, 300)
    assert "lig_b200" in mine["origin"] and "_ref" in ref["origin"]
    assert abs(mine["psnr"] - ref["psnr"]) <= 0.05, (mine["psnr"], ref["psnr"])
    # a fit that learns: far above the all-black start, and level 2 adds to level 1
    assert mine["psnr"] > mine["start"] + 10.0
    assert mine["psnr"] > mine["level1"] + 0.5
    # the checkpoint train.py saves has the reference's layout and matching content
    assert set(mine["ckpt"]) == set(ref["ckpt"]) == {"state_dict", "store_max", "store_min"}
    for sa, sb in zip(mine["ckpt"]["state_dict"], ref["ckpt"]["state_dict"]):
        assert set(sa) == set(sb)
    np.testing.assert_allclose([float(v) for v in mine["ckpt"]["store_min"]],
                               [float(v) for v in ref["ckpt"]["store_min"]], atol=1e-3)


# ------------------------------------------------------- minimal_trainer_upscale.py

def _minimal_run(arm, gt, h, w, n, iters, use_torch_upscale):
    H, W = gt.shape[2], gt.shape[3]
    with _callers.bound(arm):
        import minimal_trainer_upscale as mtu
        from optimizer import Adan
        torch.manual_seed(0)
        small = F.interpolate(gt, size=(h, w), mode="area")
        pos, rgbs, scales = mtu.init_splats_simple(n, h, w, DEV, mode="grid", image=small)
        model = mtu.Gaussian2DMinimal(pos.shape[0], h, w, DEV, positions=pos, rgbs=rgbs,
                                      scales=scales).to(DEV)
        lr, pos_scale = 0.015, max(h, w) / 512.0
        opt = Adan([{"params": model._rgb_logits, "lr": lr * 5},
                    {"params": model.means, "lr": lr * 2 * pos_scale},
                    {"params": model._cholesky, "lr": lr * pos_scale},
                    {"params": model._opacity_logits, "lr": lr}],
                   betas=(0.98, 0.92, 0.99), fused=False)
        gt_hwc = gt.squeeze(0).permute(1, 2, 0)
        params = (model.means, model._cholesky, model._rgb_logits, model._opacity_logits)
        first, losses = None, []
        for it in range(iters):
            out = model()
            img = mtu.upscale_fn(out, H, W, use_torch_upscale)
            loss = F.mse_loss(img, gt_hwc)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            if first is None:
                first = dict(img=img.detach().clone(), dx=out["dx"].detach().clone(),
                             wsum=out["wsum"].detach().clone(),
                             grads=[p.grad.detach().clone() for p in params])
            opt.step()
            losses.append(loss.item())
        with torch.no_grad():
            model.scale_to(2 * h, 2 * w)   # render the fitted set at twice the model size
            big = model()["render_hwc"].detach().clone()
        return dict(first=first, losses=losses, big=big,
                    origin=_callers.module_origin("gsplat2d"))


@pytest.mark.parametrize("use_torch_upscale", [False, True])
def test_minimal_trainer_upscale_matches_reference(use_torch_upscale):
    gt = _target(160, 192, seed=7)
    mine = _minimal_run("lig", gt, 80, 96, 2000, 8, use_torch_upscale)
    ref = _minimal_run("ref", gt, 80, 96, 2000, 8, use_torch_upscale)
    assert "lig_b200" in mine["origin"] and "_ref" in ref["origin"]
    a, b = mine["first"], ref["first"]
    for k in ("img", "dx", "wsum"):
        assert (a[k] - b[k]).abs().max().item() < 1e-5, k
    for name, ga, gb in zip(("means", "cholesky", "rgb", "opacity"), a["grads"], b["grads"]):
        assert rel_err(ga.cpu(), gb.cpu()) < 1e-4, name
    np.testing.assert_allclose(mine["losses"], ref["losses"], rtol=1e-4)
    assert (mine["big"] - ref["big"]).abs().max().item() < 1e-4
    assert mine["losses"][-1] < mine["losses"][0]
