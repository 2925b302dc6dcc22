"""Checkpoint format on the CPU: the reference's multi-level layout, level
sizes as gaussianlig.LIG derives them, and a save / load round trip."""
import torch

from lig_b200.levels import _cov_from_chol, level_sizes, load_lig, save_lig
from lig_b200.serve import GaussianSet


def _gs(n, H, W, seed, chol=True):
    g = torch.Generator().manual_seed(seed)
    return GaussianSet(torch.rand(n, 2, generator=g) * W, torch.rand(n, 3, generator=g) + 0.5,
                       torch.rand(n, 3, generator=g), H, W, cholesky=chol)


def test_level_sizes_follow_gaussianlig():
    # gaussianlig.py:23-27: H * 2^(-n_scales + s + 1)
    assert level_sizes(1000, 600, 2) == [(500, 300), (1000, 600)]
    assert level_sizes(1023, 777, 3) == [(255, 194), (511, 388), (1023, 777)]


def test_save_load_round_trip_and_reference_layout(tmp_path):
    levels = [_gs(50, 64, 80, 1), _gs(120, 128, 160, 2, chol=False)]
    p = tmp_path / "gaussian_model.pth.tar"
    save_lig(p, levels, [-0.25], [1.5])
    raw = torch.load(p, weights_only=False)
    assert set(raw) == {"state_dict", "store_max", "store_min"}
    assert raw["store_min"] == [-0.25] and raw["store_max"] == [1.5]
    for d, gs in zip(raw["state_dict"], levels):
        # the keys the reference's Gaussian2D modules load (gaussianlig.py:54-58)
        assert {"means", "cov2d", "rgbs"} <= set(d)
        assert d["means"].shape == (gs.n, 2) and d["rgbs"].shape == (gs.n, 3)
    assert torch.allclose(raw["state_dict"][0]["cov2d"], _cov_from_chol(levels[0].chol))
    m = load_lig(p, device="cpu")
    assert [(l.H, l.W) for l in m.levels] == [(64, 80), (128, 160)]
    assert m.levels[0].cholesky and not m.levels[1].cholesky
    for a, b in zip(m.levels, levels):
        assert torch.equal(a.means, b.means) and torch.equal(a.chol, b.chol)
        assert torch.equal(a.rgbs, b.rgbs)


def test_reference_file_without_sizes_needs_image_size(tmp_path):
    sd = [{"means": torch.zeros(3, 2), "cov2d": torch.ones(3, 3), "rgbs": torch.zeros(3, 3)}
          for _ in range(2)]
    p = tmp_path / "ref.pth.tar"
    torch.save({"state_dict": sd, "store_max": [torch.tensor(1.2)],
                "store_min": [torch.tensor(-0.1)]}, p)
    m = load_lig(p, device="cpu", image_hw=(200, 100))
    assert [(l.H, l.W) for l in m.levels] == [(100, 50), (200, 100)]
    assert abs(m.store_max[0] - 1.2) < 1e-6 and abs(m.store_min[0] + 0.1) < 1e-6
    try:
        load_lig(p, device="cpu")
        raise AssertionError("expected ValueError")
    except ValueError:
        pass
