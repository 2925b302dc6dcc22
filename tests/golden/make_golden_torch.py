"""Golden vectors from the reference's pure-torch upscaler (upscaler_torch.py).

Imports the reference module from its own source with TorchScript disabled
(PYTORCH_JIT=0, so @torch.jit.script returns the Python function) and gives
it a `torch` namespace whose `tensor()` places the hard-coded cuda:0 C matrix
(upscaler_torch.py:97-102) on the CPU; nothing else is changed.  Outputs and
autograd gradients go to tests/golden/torch_upscaler.npz, which pins the
oracle's align-corners upscale (tests/test_cpu_oracle_golden.py).

    python tests/golden/make_golden_torch.py [reference_root]
"""
import importlib.util
import os
import sys
import types

os.environ["PYTORCH_JIT"] = "0"
import numpy as np  # noqa: E402
import torch  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(root):
    spec = importlib.util.spec_from_file_location("ref_upscaler_torch",
                                                  os.path.join(root, "upscaler_torch.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    proxy = types.ModuleType("torch_cpu_proxy")
    proxy.__dict__.update({k: getattr(torch, k) for k in dir(torch) if not k.startswith("__")})
    proxy.tensor = lambda *a, **kw: torch.tensor(*a, **{**kw, "device": "cpu"})
    mod.torch = proxy
    return mod


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIG_REFERENCE", "/root/reference")
    mod = load_reference(root)
    g = torch.Generator().manual_seed(21)
    out = {}
    for tag, (h, w, nh, nw) in {"a": (12, 15, 35, 46), "b": (9, 9, 20, 17),
                                "c": (10, 8, 10, 8)}.items():
        planes = [torch.randn(h, w, 3, generator=g).requires_grad_() for _ in range(4)]
        up = mod.torch_gradient_aware_upscale(*planes, nh, nw)
        go = torch.randn(nh, nw, 3, generator=g)
        up.backward(go)
        out.update({f"{tag}_f": planes[0].detach().numpy(), f"{tag}_fx": planes[1].detach().numpy(),
                    f"{tag}_fy": planes[2].detach().numpy(), f"{tag}_fxy": planes[3].detach().numpy(),
                    f"{tag}_out": up.detach().numpy(), f"{tag}_go": go.numpy(),
                    f"{tag}_shape": np.array([h, w, nh, nw])})
        for k, p in zip(("gf", "gfx", "gfy", "gfxy"), planes):
            out[f"{tag}_{k}"] = p.grad.numpy()
    path = os.path.join(HERE, "torch_upscaler.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
