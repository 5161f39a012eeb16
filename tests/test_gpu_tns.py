"""Device .tns ingest (dt_tns_read / dt_tns_parse).

Checked against the reference's own read_data<double> (src/read_data.cpp:36-129,
compiled in the oracle) on files it can read, and against Python's correctly
rounded float() for the value formats the reference cannot read (signs,
exponents, long mantissas).  Indices, dims and value bits must match exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _coo(shape, nnz, seed):
    rng = np.random.default_rng(seed)
    idx = [rng.integers(0, s, nnz) for s in shape]
    return idx, rng


def _lines(idx, strs):
    return "".join(" ".join(str(int(i[e]) + 1) for i in idx) + " " + strs[e] + "\n"
                   for e in range(len(strs)))


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("shape,nnz", [((30, 20, 10), 5000), ((7, 9, 11, 13), 3000)])
def test_matches_reference_reader(ctx, oracle_ref, tmp_path, shape, nnz):
    idx, rng = _coo(shape, nnz, 7 + len(shape))
    # read_double takes digits and '.' only (read_data.cpp:24-33).
    strs = [f"{v:.6f}" for v in rng.lognormal(0.0, 2.0, nnz)]
    path = str(tmp_path / "a.tns")
    with open(path, "w") as f:
        f.write(_lines(idx, strs))
    ri, rv, rd = oracle_ref.read_tns(path)
    gi, gv, gd = ctx.read_tns(path)
    assert len(gi) == len(ri) == len(shape)
    for m in range(len(shape)):
        np.testing.assert_array_equal(gi[m], ri[m])
    np.testing.assert_array_equal(_bits(gv), _bits(rv))
    np.testing.assert_array_equal(gd, rd)


def test_values_are_correctly_rounded(ctx):
    rng = np.random.default_rng(3)
    n = 200000
    mag = 10.0 ** rng.uniform(-280, 280, n)
    v = mag * rng.choice([-1.0, 1.0], n)
    fmts = ["%.17g", "%.6e", "%.3f", "%.12g", "%.20e", "%.1e"]
    strs = [fmts[e % len(fmts)] % v[e] for e in range(n)]
    strs += ["0", "-0.0", "+3", ".5", "5.", "1e5", "1E-5", "123456789012345678901234",
             "0.000000000000000000000001234", "9007199254740993", "4.9406564584124654e-300",
             "1.7976931348623157e+280", "2.2250738585072014e-280", "00012.5000",
             "0.001e330", "1e400", "-1e-400"]
    idx = [np.arange(len(strs)) % 5, np.arange(len(strs)) % 3]
    gi, gv, gd = ctx.read_tns(data=_lines(idx, strs).encode())
    want = np.array([float(s) for s in strs])
    bad = np.nonzero(_bits(gv) != _bits(want))[0]
    assert bad.size == 0, [(strs[b], repr(gv[b]), repr(want[b])) for b in bad[:5]]
    np.testing.assert_array_equal(gi[0], idx[0])
    np.testing.assert_array_equal(gd, [5, 3])


def test_blank_lines_tabs_crlf_and_no_final_newline(ctx):
    text = "\n1 2\t3 1.5\r\n\n   \n2 1 1 -2.5e-3\r\n3  3 2 7"
    gi, gv, gd = ctx.read_tns(data=text.encode())
    np.testing.assert_array_equal(gi[0], [0, 1, 2])
    np.testing.assert_array_equal(gi[1], [1, 0, 2])
    np.testing.assert_array_equal(gi[2], [2, 0, 1])
    np.testing.assert_array_equal(_bits(gv), _bits([1.5, -2.5e-3, 7.0]))
    np.testing.assert_array_equal(gd, [3, 3, 3])


@pytest.mark.parametrize("text,line,word", [
    ("1 1 1 1.0\n2 2 2 2.0\n3 3 1.0\n", 3, "indices"),
    ("1 1 1 1.0\n0 2 2 2.0\n", 2, "1-based"),
    ("1 1 1 1.0\n2 2 2 x2.0\n", 2, "number"),
    ("1 1 1 1.0\n2 2 2 2.0 5\n", 2, "indices"),
])
def test_malformed_lines_are_rejected(ctx, text, line, word):
    from diana_tucker_b200 import DTError
    with pytest.raises(DTError) as e:
        ctx.read_tns(data=text.encode())
    assert e.value.code == 1
    assert f"line {line}" in str(e.value) and word in str(e.value)


def test_many_chunks_and_sptensor_from_tns(ctx, oracle_sparse):
    from diana_tucker_b200 import datasets
    idx, vals, shape = datasets.sparse_zipf((5000, 3000, 2000), 400000, alpha=1.1, seed=9)
    strs = [repr(float(x)) for x in vals]
    data = _lines(idx, strs).encode()
    assert len(data) > 8 * 64 * 1024
    gi, gv, gd = ctx.read_tns(data=data)
    for m in range(3):
        np.testing.assert_array_equal(gi[m], idx[m])
    np.testing.assert_array_equal(_bits(gv), _bits(vals))
    np.testing.assert_array_equal(gd, [int(i.max()) + 1 for i in idx])
    # The sparse tensor built from the device copy equals one built from the
    # host arrays: same TTMc, bit for bit.
    R = (8, 8, 8)
    Ut = datasets.random_orthonormal_transposed(list(gd), R, 2)
    a = ctx.sptensor_from_tns(data=data)
    b = ctx.sptensor(idx, vals, list(gd))
    for mode in range(3):
        np.testing.assert_array_equal(a.ttmc_mTR(Ut, R, mode), b.ttmc_mTR(Ut, R, mode))
    a.close()
    b.close()
