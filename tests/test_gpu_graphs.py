"""Dense HOOI through the context's cached plans and captured sweep graphs.

On a stream other than the legacy default stream, dt_hooi_dense keeps its
buffers between calls with the same shapes and ranks and replays each sweep
from a captured CUDA graph; the tensor-core path's split sweeps run as one
graph whose WHILE node repeats a sweep and its stop test on the device.  The
results must equal direct launches (legacy stream, no graph, the host
deciding after each sweep) to FP64 rounding: the same kernels run in the same
order.  Tolerance: 1e-12 relative (norm-wise)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _tensor(shape, ranks, seed):
    from diana_tucker_b200 import datasets
    return datasets.tucker_dense(shape, ranks, noise_var=1e-4, seed=seed, dtype=np.float32)


def _run(ctx, Xt, ranks, precision, shape):
    G, U, rep = ctx.hooi_dense(Xt, ranks, init="randn", seed=3, max_sweeps=6, tol=1e-10,
                               precision=precision, shape=shape)
    return G, U, rep


@pytest.mark.parametrize("prec", ["fp64", "bf16x2"])
def test_graph_replay_matches_direct_launches(ctx, prec):
    import torch

    from diana_tucker_b200 import DT_PREC_BF16X2, DT_PREC_FP64
    precision = DT_PREC_FP64 if prec == "fp64" else DT_PREC_BF16X2
    # Shapes every tensor-core contraction of the dimension tree accepts.
    shape, ranks = (96, 80, 72), (8, 8, 8)
    X = _tensor(shape, ranks, 41)
    flat = np.ascontiguousarray(X.reshape(-1, order="F"))
    Xd = torch.from_numpy(flat).cuda()
    if precision == DT_PREC_FP64:
        Xd = Xd.double()
    # Direct launches: torch's legacy default stream takes no graphs.
    G0, U0, r0 = _run(ctx, Xd, ranks, precision, shape)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        G1, U1, r1 = _run(ctx, Xd, ranks, precision, shape)   # builds the plan, captures
        G2, U2, r2 = _run(ctx, Xd, ranks, precision, shape)   # replays
        # A different shape replaces the plan; the first shape then rebuilds it.
        Y = torch.from_numpy(np.ascontiguousarray(
            _tensor((64, 64, 48), (8, 8, 8), 42).reshape(-1, order="F"))).cuda()
        if precision == DT_PREC_FP64:
            Y = Y.double()
        _run(ctx, Y, (8, 8, 8), precision, (64, 64, 48))
        G3, U3, r3 = _run(ctx, Xd, ranks, precision, shape)
    torch.cuda.synchronize()
    assert r0["precision_used"] == precision
    for G, U, r in ((G1, U1, r1), (G2, U2, r2), (G3, U3, r3)):
        assert r["precision_used"] == precision
        assert r["sweeps"] == r0["sweeps"]
        assert abs(r["residual"] - r0["residual"]) <= 1e-12
        # The split sweeps run as one device-side loop on a capturable stream:
        # each sweep adds the loop's stop-test kernel.
        extra = r["sweeps"] if precision == DT_PREC_BF16X2 else 0
        # A plan that has drawn this seed's initial factors copies them (one
        # copy launch) instead of orthonormalising new draws (one launch).
        assert r["kernel_launches"] - extra == r0["kernel_launches"]
        assert _nrel(G, G0) < 1e-12
        for n in range(3):
            assert _nrel(U[n], U0[n]) < 1e-12
