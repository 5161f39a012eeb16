"""Runs the dense HOOI of the 96^4 rank-16 benchmark tensor a few times, for
profilers (ncu, compute-sanitizer): one line per call with its wall time,
device time, sweeps, residual and kernel launches.

    python -m diana_tucker_b200.hooi_profile [xh|x2|bf16|fp64] [calls]
    python -m diana_tucker_b200.hooi_profile batched [count]

The first call builds the plan and captures the sweep graphs; later calls
replay them, as in the bench.  `batched` runs the batched HOOI three times on
the first `count` tensors of the bench's batch (seed 3; 10 sweeps of five
ALS_ steps, 512 threads per CTA, pairs packed), X resident.
"""
from __future__ import annotations

import sys
import time


def main(argv=None):
    import numpy as np
    import torch

    from . import (DT_PREC_BF16, DT_PREC_BF16X2, DT_PREC_BF16XH, DT_PREC_FP64, Context,
                   datasets)
    argv = sys.argv[1:] if argv is None else argv
    name = argv[0] if argv else "xh"
    if name == "batched":
        return batched(int(argv[1]) if len(argv) > 1 else 600)
    prec = {"xh": DT_PREC_BF16XH, "x2": DT_PREC_BF16X2, "bf16": DT_PREC_BF16,
            "fp64": DT_PREC_FP64}[name]
    calls = int(argv[1]) if len(argv) > 1 else 5
    ctx = Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    X = datasets.dense_96x4_fp32()
    Xd = torch.from_numpy(np.ascontiguousarray(X.reshape(-1, order="F"))).cuda()
    if prec == DT_PREC_FP64:
        Xd = Xd.double()
    kw = dict(init="randn", seed=1, max_sweeps=30, tol=1e-9, shape=X.shape,
              inner_iters=5 if prec == DT_PREC_FP64 else 2, precision=prec, device_out=True)
    for i in range(calls):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, rep = ctx.hooi_dense(Xd, (16,) * 4, **kw)
        torch.cuda.synchronize()
        print(f"call {i}: {(time.perf_counter() - t0) * 1e3:.3f} ms wall, device "
              f"{rep['device_ms']:.3f} ms, sweeps {rep['sweeps']}, residual "
              f"{rep['residual']:.12f}, launches {rep['kernel_launches']}", flush=True)
    ctx.close()


def batched(count):
    import numpy as np
    import torch

    from . import Context, datasets
    ctx = Context(0)
    items = datasets.batched_small(count=count, seed=3)
    rng = np.random.default_rng(103)
    U0 = [[np.linalg.qr(rng.standard_normal((X.shape[k], r[k])))[0] for k in range(3)]
          for X, r in items]
    pk = ctx.pack_batched([X for X, _ in items], [r for _, r in items], U0)
    dev = torch.device("cuda", 0)
    Xd = torch.from_numpy(pk["X"]).to(dev)
    U0d = torch.from_numpy(pk["U"]).to(dev)
    Ud = U0d.clone()
    Gd = torch.zeros(pk["g_size"], dtype=torch.float64, device=dev)
    Ed = torch.zeros(pk["count"], dtype=torch.float64, device=dev)
    for i in range(3):
        Ud.copy_(U0d)
        rep = ctx.hooi_batched_packed(pk, Ud, Gd, Ed, X=Xd, sweeps=10, inner_iters=5,
                                      block_threads=512)
        print(f"call {i}: device {rep['device_ms']:.3f} ms, items {rep['items']}, "
              f"pack {rep['pack']}", flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
