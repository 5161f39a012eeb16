"""The Python host layer's output buffers for device results (no GPU needed:
the same views are built on the CPU).

Context.hooi_dense(..., device_out=True) hands the library one float64
allocation holding the core and then every factor; each is returned as a
column-major view, the layout the C ABI writes (dt_cuda.h: tensors are
column-major, a factor U_n is I_n x R_n column-major).
"""
import numpy as np
import pytest
import torch

from diana_tucker_b200 import _column_major_outputs


@pytest.mark.parametrize("shape,ranks", [((7, 8, 9), (3, 4, 5)), ((96,) * 4, (16,) * 4),
                                         ((5,), (2,)), ((4, 6), (4, 1))])
def test_core_and_factors_are_column_major_views_of_one_buffer(shape, ranks):
    G, U = _column_major_outputs(shape, ranks, True, True, "cpu")
    N = len(shape)
    base = G.data_ptr()
    gsize = int(np.prod(ranks))
    # The core: shape R, strides 1, R_0, R_0 R_1, ...
    assert tuple(G.shape) == tuple(ranks)
    assert G.stride() == tuple(int(np.prod(ranks[:m])) for m in range(N))
    # The factors follow the core back to back, each I_n x R_n column-major.
    off = gsize
    for n in range(N):
        assert tuple(U[n].shape) == (shape[n], ranks[n])
        assert U[n].stride() == (1, shape[n])
        assert U[n].data_ptr() == base + 8 * off
        assert U[n].untyped_storage().data_ptr() == G.untyped_storage().data_ptr()
        off += shape[n] * ranks[n]
    assert G.untyped_storage().nbytes() == 8 * off
    # Writing the flat buffer in the library's order reads back element by element.
    flat = torch.arange(off, dtype=torch.float64)
    G.untyped_storage().copy_(flat.untyped_storage())
    idx = tuple(r - 1 for r in ranks)
    lin = sum(i * s for i, s in zip(idx, G.stride()))
    assert G[idx].item() == lin
    off = gsize
    for n in range(N):
        i, r = shape[n] - 1, ranks[n] - 1
        assert U[n][i, r].item() == off + i + shape[n] * r
        off += shape[n] * ranks[n]


def test_outputs_not_asked_for_are_not_allocated():
    G, U = _column_major_outputs((7, 8, 9), (3, 4, 5), False, True, "cpu")
    assert G is None and U[0].data_ptr() == U[0].untyped_storage().data_ptr()
    G, U = _column_major_outputs((7, 8, 9), (3, 4, 5), True, False, "cpu")
    assert U is None and G.untyped_storage().nbytes() == 8 * 60
    G, U = _column_major_outputs((7, 8, 9), (3, 4, 5), False, False, "cpu")
    assert G is None and U is None
