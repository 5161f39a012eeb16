"""Dense HOOI results returned as CUDA tensors (device_out=True: the core and
the factors as column-major views of one device allocation, filled by one
copy launch) equal the same call's results copied to host arrays."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("prec", ["FP64", "BF16XH"])
def test_device_outputs_equal_host_outputs(ctx, prec):
    import torch

    import diana_tucker_b200 as dtb
    precision = getattr(dtb, "DT_PREC_" + prec)
    rng = np.random.default_rng(7)
    shape, ranks = (64, 48, 40), (8, 8, 8)
    X = rng.standard_normal(shape).astype(np.float32)
    x = torch.from_numpy(np.ascontiguousarray(X.reshape(-1, order="F"))).cuda()
    if prec == "FP64":
        x = x.double()
    kw = dict(precision=precision, max_sweeps=3, inner_iters=2, shape=shape)
    Gh, Uh, rh = ctx.hooi_dense(x, ranks, **kw)
    Gd, Ud, rd = ctx.hooi_dense(x, ranks, device_out=True, **kw)
    torch.cuda.synchronize()
    assert Gd.is_cuda and tuple(Gd.shape) == ranks and Gd.stride() == (1, 8, 64)
    assert rd["sweeps"] == rh["sweeps"]
    assert abs(rd["residual"] - rh["residual"]) <= 1e-12
    assert _rel(Gd.cpu().numpy(), Gh) <= 1e-12
    for n in range(3):
        assert Ud[n].is_cuda and tuple(Ud[n].shape) == (shape[n], ranks[n])
        assert Ud[n].stride() == (1, shape[n])
        assert _rel(Ud[n].cpu().numpy(), Uh[n]) <= 1e-12
