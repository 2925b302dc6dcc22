"""Generate golden vectors from the reference's own CUDA kernels.

Runs on a GPU machine with oracle/_ref/libgsplat2d_ref.so (built from the
reference sources by `make -C oracle ref`).  Writes one compressed .npz per
case holding the seeded inputs and every reference output; the CPU test
tests/test_cpu_oracle_golden.py checks the C oracle against them.

    python tests/golden/make_golden_ref.py [out_dir]   (default tests/golden)
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from tests._scene import scene  # noqa: E402

CASES = {
    # name: (n, H, W, B, diag, opacity range)
    "b16_op": (170, 40, 52, 16, (0.5, 4.0), (0.0, 1.0)),
    "b12_op": (120, 36, 45, 12, (0.3, 3.0), (0.1, 0.95)),
    "b8_noop": (100, 32, 32, 8, (0.5, 3.0), None),
}
UP_H, UP_W = 14, 18  # source planes of the upscale cases


def np_(t):
    return None if t is None else t.detach().cpu().numpy()


def case(name, n, H, W, B, diag, opac, out_dir):
    means, L, colors, op = scene(n, H, W, diag=diag, opac=opac, seed=11)
    d = dict(H=H, W=W, B=B, means=np_(means), chol=np_(L), colors=np_(colors))
    if op is not None:
        d["opac"] = np_(op)
    xys, ext, con, cnt = ref.project_fwd(L, means, op, H, W, B, True)
    d.update(xys=np_(xys), extents=np_(ext), conics=np_(con), counts=np_(cnt))
    bn = ref.bin_and_sort(xys, ext, cnt, H, W, B)
    d.update(cum=np_(bn.cum_tiles_hit), isect_ids=np_(bn.isect_ids), gids=np_(bn.gaussian_ids),
             isect_sorted=np_(bn.isect_ids_sorted), gid_sorted=np_(bn.gaussian_ids_sorted),
             tile_bins=np_(bn.tile_bins))
    g = torch.Generator().manual_seed(3)
    cot = [torch.randn(s, generator=g).cuda() for s in [(H, W, 3), (H, W), (H, W, 3), (H, W, 3),
                                                        (H, W, 3)]]
    d.update(v_img=np_(cot[0]), v_wsum=np_(cot[1]), v_dx=np_(cot[2]), v_dy=np_(cot[3]),
             v_dxy=np_(cot[4]))
    for ga in (False, True):
        tag = "ga" if ga else "sum"
        r = ref.raster_fwd(H, W, B, bn, xys, con, colors, op, ga)
        for k in ("img", "wsum", "final_idx", "dx", "dy", "dxy"):
            if r[k] is not None:
                d[f"{tag}_{k}"] = np_(r[k])
        vd = cot[2:] if ga else [None] * 3
        rg = ref.raster_bwd(H, W, B, bn, xys, con, colors, op, r["final_idx"], cot[0], cot[1],
                            *vd)
        for k, v in rg.items():
            if v is not None:
                d[f"{tag}_{k}"] = np_(v)
    v_xy = torch.randn(n, 2, generator=g).cuda()
    v_con = torch.randn(n, 3, generator=g).cuda()
    v_in3, v_mean = ref.project_bwd(ext, L, con, v_xy, v_con, True)
    d.update(pb_v_xy=np_(v_xy), pb_v_conic=np_(v_con), pb_v_chol=np_(v_in3), pb_v_mean=np_(v_mean))
    # upscale: render planes -> 3x and a ROI crop
    planes = [torch.randn(UP_H, UP_W, 3, generator=g).cuda() for _ in range(4)]
    d.update(up_f=np_(planes[0]), up_fx=np_(planes[1]), up_fy=np_(planes[2]), up_fxy=np_(planes[3]))
    roi = (3.0, 2.0, float(UP_W) - 4.5, float(UP_H) - 1.0)
    for tag, r_, dh, dw in (("full", None, 3 * UP_H, 3 * UP_W), ("roi", roi, 2 * UP_H, 2 * UP_W)):
        d[f"up_{tag}_out"] = np_(ref.upscale_fwd(*planes, dh, dw, r_))
        go = torch.randn(dh, dw, 3, generator=g).cuda()
        d[f"up_{tag}_g"] = np_(go)
        for k, v in zip(("gf", "gfx", "gfy", "gfxy"), ref.upscale_bwd(go, UP_H, UP_W, r_)):
            d[f"up_{tag}_{k}"] = np_(v)
    d["up_roi"] = np.array(roi)
    path = os.path.join(out_dir, f"ref_{name}.npz")
    np.savez_compressed(path, **{k: v for k, v in d.items() if v is not None})
    print(path, os.path.getsize(path))


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden")
    os.makedirs(out_dir, exist_ok=True)
    for name, c in CASES.items():
        case(name, *c, out_dir)


if __name__ == "__main__":
    main()
