"""Summary profiler (dt_summary_*): the reference's Summary::print_summary table
(src/summary.cpp:100-206) over device-timed ranges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(table):
    """{name: (time, counted, number, avg, gflops, gbs)} from the table text."""
    out, name = {}, None
    for line in table.splitlines():
        if not line.startswith("| "):
            continue
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) == 2 and cells[0]:
            name = cells[0]
        elif len(cells) == 3 and not cells[0] and name is not None:
            f, g = cells[1].split(), cells[2].split()
            out[name] = (float(f[0]), f[1], int(f[2]), float(f[3]), float(g[0]), float(g[1]))
            name = None
    return out


def test_summary_table_counts_hooi_and_ttmc(ctx):
    from diana_tucker_b200 import datasets
    X = datasets.tucker_dense((40, 32, 24), (5, 4, 3), noise_var=1e-4, seed=1)
    idx, vals, shape = datasets.sparse_zipf((500, 300, 200), 5000, seed=5)
    Ut = datasets.random_orthonormal_transposed(shape, (8, 8, 8), 6)
    sp = ctx.sptensor(idx, vals, shape)
    ctx.summary_enable(True)
    try:
        _, _, rep = ctx.hooi_dense(X, (5, 4, 3), init="randn", max_sweeps=3)
        ctx.ttm(X, np.ones((2, 32)), 1)
        sp.hooi((8, 8, 8), 2, Ut)
        table = ctx.summary_table()
    finally:
        ctx.summary_enable(False)
        sp.close()
    assert "Time C.(%)" in table and "Bandw.(GB/s)" in table
    rows = _rows(table)
    assert rows["Algorithm::Tucker::HOOI_ALS()"][2] == 1
    assert rows["HOOI sweep (FP64)"][2] == rep["sweeps"] == 3
    assert rows["Function::ttm()"][2] == 1
    assert rows["Algorithm::SpTucker::Sp_HOOI_ALS()"][2] == 1
    # 2 sweeps x 3 modes + the final core's TTMc.
    assert rows["Function::ttmc()"][2] == 7
    assert rows["Function::ttmc()"][1] == "Kernel"
    for name, (t, counted, n, avg, gf, gb) in rows.items():
        assert t > 0 and n >= 1 and abs(avg - t / n) <= 1e-6 * max(1.0, t)
    # Nested ranges count towards their caller: HOOI_ALS spends its time in
    # its sweeps, and {Main} holds everything.
    assert float(rows["Algorithm::Tucker::HOOI_ALS()"][1]) > 50.0
    assert rows["{Main}"][0] >= rows["Algorithm::Tucker::HOOI_ALS()"][0]
