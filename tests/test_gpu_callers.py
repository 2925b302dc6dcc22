"""LIG's own training code, unmodified, on this library vs on the reference.

Each test runs the reference's gaussianlig.py, train.py or
minimal_trainer_upscale.py (bytecode of the unmodified files; see
tests/_callers.py) twice in this process: once with `gsplat2d` /
`upscaler_torch` resolving to this library through
lig_b200.install_gsplat2d(), once with them resolving to the reference's own
gsplat2d package on the reference's kernels.  Same seeds, same target; the
comparison is on what LIG's code computes: renders (1e-5), gradients
(1e-4 relative) and the optimizer's moments (5e-4 relative), with the two
arms in lockstep (each iteration starts both from the reference arm's
parameters and optimizer state), and the PSNR of free-running fits (0.05 dB).

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


# ------------------------------------------------------------------- lockstep
# A fit's trajectory is chaotic under Adam / Adan: their first steps move each
# parameter by about lr * sign(gradient), so a gradient at rounding-noise
# level (the backward's float atomics add in a run-dependent order, in the
# reference as here) can take either sign and the two runs part ways.  The
# per-iteration comparisons therefore run the two arms in lockstep: before
# each iteration this library's model takes the reference model's parameters
# and optimizer state (by value), then both run the same unmodified step.
# End-of-fit agreement of free-running fits is the PSNR test on train.py.

def _sync(dst_params, dst_opt, src_params, src_opt):
    """dst takes src's parameters and optimizer state, by value."""
    with torch.no_grad():
        for a, b in zip(dst_params, src_params):
            a.copy_(b)
            st = src_opt.state.get(b, {})
            dst_opt.state[a] = {k: (v.clone() if torch.is_tensor(v) else v)
                                for k, v in st.items()}


def _opt_state(opt, params):
    return [{k: v.detach().clone() for k, v in opt.state[p].items()
             if torch.is_tensor(v) and v.numel() > 1} for p in params]


def _assert_opt_state_close(sa, sb, tol):
    for da, db in zip(sa, sb):
        assert set(da) == set(db)
        for k in da:
            assert rel_err(da[k].cpu(), db[k].cpu()) < tol, k


# ----------------------------------------------------------------- gaussianlig.py

def _gaussianlig_model(arm, H, W, n):
    with _callers.bound(arm):
        import gaussianlig
        torch.manual_seed(0)
        m = gaussianlig.Gaussian2D(loss_type="L2", opt_type="adam", num_points=n, H=H, W=W,
                                   BLOCK_H=16, BLOCK_W=16, device=DEV, lr=0.018)
        return m, _callers.module_origin("gsplat2d")


def _gaussianlig_step(arm, m, gt):
    """One Gaussian2D.train_iter (gaussianlig.py:99-111), recording the
    gradients the optimizer sees and its state after the step."""
    params = (m.means, m.cov2d, m.rgbs)
    rec = {}
    step = m.optimizer.step

    def recording_step(*a, **k):
        rec["grads"] = [p.grad.detach().clone() for p in params]
        out = step(*a, **k)
        rec["state"] = _opt_state(m.optimizer, params)
        return out

    m.optimizer.step = recording_step
    try:
        with _callers.bound(arm):
            loss, psnr = m.train_iter(gt)
    finally:
        m.optimizer.step = step
    rec["loss"], rec["psnr"] = float(loss), psnr
    return rec


def test_gaussianlig_train_iter_matches_reference():
    H, W, n = 96, 128, 3000
    gt = _target(H, W)
    mine, o_mine = _gaussianlig_model("lig", H, W, n)
    ref, o_ref = _gaussianlig_model("ref", H, W, n)
    assert "lig_b200" in o_mine and "_ref" in o_ref
    pm, pr = (mine.means, mine.cov2d, mine.rgbs), (ref.means, ref.cov2d, ref.rgbs)
    for a, b in zip(pm, pr):
        assert torch.equal(a, b)
    psnrs = []
    for it in range(10):
        _sync(pm, mine.optimizer, pr, ref.optimizer)
        a = _gaussianlig_step("lig", mine, gt)
        b = _gaussianlig_step("ref", ref, gt)
        for name, ga, gb in zip(("means", "cov2d", "rgbs"), a["grads"], b["grads"]):
            assert rel_err(ga.cpu(), gb.cpu()) < 1e-4, (it, name)
        assert abs(a["loss"] - b["loss"]) <= 1e-5 * abs(b["loss"]), it
        assert abs(a["psnr"] - b["psnr"]) <= 1e-4, it
        _assert_opt_state_close(a["state"], b["state"], 5e-4)   # Adam's moments
        psnrs.append(b["psnr"])
    _sync(pm, mine.optimizer, pr, ref.optimizer)
    with torch.no_grad():
        with _callers.bound("lig"):
            r_mine = mine.forward()["render"].detach().clone()
        with _callers.bound("ref"):
            r_ref = ref.forward()["render"].detach().clone()
    assert (r_mine - r_ref).abs().max().item() < 1e-5
    assert psnrs[-1] > psnrs[0] + 1.0   # the fit learns


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
    """train.py's free-running two-level fit, three runs per arm, medians
    compared.  The fit is chaotic for both implementations: any two runs,
    the reference against itself included, part by more than 1e-3 dB within
    about 30 of the 300 iterations (the backward's float atomics add in a
    run-dependent order), and the final PSNR has a heavy tail because level 2
    fits a residual min-max-normalised by level 1's extreme pixels, so one
    run in several can land far from the rest (+1.4 dB was seen).  The
    median of three is robust to one such run on either side."""
    from PIL import Image
    gt = _target(256, 256, seed=6)
    arr = (gt[0].permute(1, 2, 0).cpu().numpy() * 255).round().astype(np.uint8)
    png = tmp_path / "synthetic_0001.png"
    Image.fromarray(arr).save(png)
    runs = {"lig": [], "ref": []}
    for rep in range(3):
        for arm in ("lig", "ref"):
            runs[arm].append(_train_py_run(arm, png, tmp_path / f"{arm}{rep}", 12000, 300))
    mine = sorted(runs["lig"], key=lambda r: r["psnr"])[1]
    ref = sorted(runs["ref"], key=lambda r: r["psnr"])[1]
    assert all("lig_b200" in r["origin"] for r in runs["lig"])
    assert all("_ref" in r["origin"] for r in runs["ref"])
    assert abs(mine["psnr"] - ref["psnr"]) <= 0.05, (
        [r["psnr"] for r in runs["lig"]], [r["psnr"] for r in runs["ref"]])
    # a fit that learns: far above the all-black start, and level 2 adds to level 1
    assert mine["psnr"] > mine["start"] + 10.0
    assert mine["psnr"] > mine["level1"] + 0.5
    # the checkpoint train.py saves has the reference's layout and matching content
    assert set(mine["ckpt"]) == set(ref["ckpt"]) == {"state_dict", "store_max", "store_min"}
    for sa, sb in zip(mine["ckpt"]["state_dict"], ref["ckpt"]["state_dict"]):
        assert set(sa) == set(sb)
    np.testing.assert_allclose([float(v) for v in mine["ckpt"]["store_min"]],
                               [float(v) for v in ref["ckpt"]["store_min"]], atol=1e-2)


# ------------------------------------------------------- minimal_trainer_upscale.py

def _minimal_setup(arm, gt, h, w, n):
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
        params = (model.means, model._cholesky, model._rgb_logits, model._opacity_logits)
        return dict(mtu=mtu, model=model, opt=opt, params=params,
                    origin=_callers.module_origin("gsplat2d"))


def _minimal_step(arm, run, gt, use_torch_upscale):
    """Gaussian2DMinimal.forward + upscale_fn (minimal_trainer_upscale.py:
    124-170), the L2 loss, backward and one Adan step."""
    H, W = gt.shape[2], gt.shape[3]
    gt_hwc = gt.squeeze(0).permute(1, 2, 0)
    model, opt, params = run["model"], run["opt"], run["params"]
    with _callers.bound(arm):
        out = model()
        img = run["mtu"].upscale_fn(out, H, W, use_torch_upscale)
        loss = F.mse_loss(img, gt_hwc)
        opt.zero_grad(set_to_none=True)
        loss.backward()
        rec = dict(img=img.detach().clone(), dx=out["dx"].detach().clone(),
                   wsum=out["wsum"].detach().clone(),
                   grads=[p.grad.detach().clone() for p in params], loss=loss.item())
        opt.step()
    rec["state"] = _opt_state(opt, params)
    return rec


@pytest.mark.parametrize("use_torch_upscale", [False, True])
def test_minimal_trainer_upscale_matches_reference(use_torch_upscale):
    gt = _target(160, 192, seed=7)
    h, w, n = 80, 96, 2000
    mine = _minimal_setup("lig", gt, h, w, n)
    ref = _minimal_setup("ref", gt, h, w, n)
    assert "lig_b200" in mine["origin"] and "_ref" in ref["origin"]
    losses = []
    for it in range(8):
        _sync(mine["params"], mine["opt"], ref["params"], ref["opt"])
        a = _minimal_step("lig", mine, gt, use_torch_upscale)
        b = _minimal_step("ref", ref, gt, use_torch_upscale)
        for k in ("img", "dx", "wsum"):
            assert (a[k] - b[k]).abs().max().item() < 1e-5, (it, k)
        for name, ga, gb in zip(("means", "cholesky", "rgb", "opacity"), a["grads"], b["grads"]):
            assert rel_err(ga.cpu(), gb.cpu()) < 1e-4, (it, name)
        assert abs(a["loss"] - b["loss"]) <= 1e-5 * abs(b["loss"]), it
        _assert_opt_state_close(a["state"], b["state"], 5e-4)   # Adan's moments
        losses.append(b["loss"])
    _sync(mine["params"], mine["opt"], ref["params"], ref["opt"])
    big = []
    for arm, run in (("lig", mine), ("ref", ref)):
        with torch.no_grad(), _callers.bound(arm):
            run["model"].scale_to(2 * h, 2 * w)   # the fitted set at twice the model size
            big.append(run["model"]()["render_hwc"].detach().clone())
    assert (big[0] - big[1]).abs().max().item() < 1e-5
    assert losses[-1] < losses[0]
