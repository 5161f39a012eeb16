"""diana_tucker_b200 -- DIANA-Tucker's HOOI-ALS hot path on B200 (sm_100a).

Python host layer over the C ABI of ``libdt_cuda.so`` (include/dt_cuda.h).
Every computation runs in the CUDA library; this module only moves buffers:
numpy arrays are passed as host pointers (the library stages them), torch
CUDA tensors are passed as device pointers on torch's current stream.

The C++ drop-in for the reference's own API (``Tensor<Ty>``, ``SpTensor<Ty>``,
``Function::ttm``, ``Algorithm::Tucker::HOOI_ALS`` ...) lives in
``cpp/include/diana``.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from . import _lib
from ._lib import (DT_INIT_GIVEN, DT_INIT_HOSVD, DT_INIT_RANDN_LIBC, DT_PREC_BF16,
                   DT_PREC_BF16X2, DT_PREC_BF16XH, DT_PREC_FP64, DTError, HooiOpts, HooiReport)

__all__ = ["Context", "SpTensor", "DTError", "DT_PREC_FP64", "DT_PREC_BF16", "DT_PREC_BF16X2",
           "DT_PREC_BF16XH",
           "DT_INIT_RANDN_LIBC", "DT_INIT_HOSVD", "DT_INIT_GIVEN"]


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _column_major_outputs(shape, ranks, want_core, want_factors, device):
    """The core (ranks, column-major) and the factors (shape[n] x ranks[n],
    column-major) as float64 views of one uninitialised torch allocation on
    `device`, the core first, then U_0, U_1, ...  The library writes every
    entry.  Returns (G or None, [U_n] or None)."""
    import torch
    shape = [int(i) for i in shape]
    ranks = [int(r) for r in ranks]
    gsize = math.prod(ranks) if want_core else 0
    usizes = [i * r for i, r in zip(shape, ranks)] if want_factors else []
    buf = torch.empty(gsize + sum(usizes), dtype=torch.float64, device=device)
    # One as_strided view each (a view op costs a few microseconds of host
    # time per call): column-major strides 1, R_0, R_0 R_1, ...
    G = None
    if want_core:
        strides, st = [], 1
        for r in ranks:
            strides.append(st)
            st *= r
        G = buf.as_strided(ranks, strides, 0)
    U, off = ([] if want_factors else None), gsize
    for i, r, sz in zip(shape, ranks, usizes):
        U.append(buf.as_strided((i, r), (1, i), off))
        off += sz
    return G, U


def _shape_arr(shape):
    return np.ascontiguousarray(np.asarray(shape, dtype=np.int64))


def _i64p(a: np.ndarray):
    return a.ctypes.data_as(_lib.c_i64p)


class _Buf:
    """A caller buffer as (pointer, keep-alive owner)."""

    def __init__(self, x, dtype=np.float64, fortran=True, writable=False):
        self.torch = _is_torch(x)
        if self.torch:
            import torch
            tdt = torch.float64 if dtype == np.float64 else torch.float32
            if x.dtype != tdt:
                raise TypeError(f"expected {tdt}, got {x.dtype}")
            self.obj = x
            self.ptr = ctypes.c_void_p(x.data_ptr())
        else:
            a = np.asarray(x, dtype=dtype)
            a = np.asfortranarray(a) if fortran else np.ascontiguousarray(a)
            if writable and a is not x:
                a = a.copy(order="F" if fortran else "C")
            self.obj = a
            self.ptr = ctypes.c_void_p(a.ctypes.data)


def _alloc_like(ref_is_torch, shape, dtype=np.float64, device=None):
    if ref_is_torch:
        import torch
        # Column-major storage: allocate the reversed shape C-contiguous and
        # expose it transposed, so data_ptr() holds the col-major layout.
        t = torch.empty(tuple(reversed(shape)), dtype=torch.float64, device=device)
        return t.permute(*reversed(range(len(shape)))) if len(shape) > 1 else t
    return np.zeros(shape, dtype=dtype, order="F")


_CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


class Context:
    """A dt_ctx bound to one GPU (dt_ctx_create)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self.lib.dt_ctx_create(device, ctypes.byref(h)))
        self.h = h
        self.device = device
        self._torch_stream = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.dt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- stream plumbing --------------------------------------------------
    def _bind(self, *objs):
        """Runs on torch's current stream when torch tensors are involved."""
        if any(_is_torch(o) for o in objs):
            import torch
            s = torch.cuda.current_stream(self.device).cuda_stream
            # Handle 0 is torch's legacy default stream; NULL would select the
            # context's own (non-blocking) stream, so pass cudaStreamLegacy.
            if s == 0:
                s = _CUDA_STREAM_LEGACY
            if s != self._torch_stream:
                _lib.check(self.lib.dt_ctx_set_stream(self.h, ctypes.c_void_p(s)))
                self._torch_stream = s
        elif self._torch_stream is not None:
            _lib.check(self.lib.dt_ctx_set_stream(self.h, None))
            self._torch_stream = None

    def synchronize(self):
        _lib.check(self.lib.dt_ctx_synchronize(self.h))

    def kernel_launches(self) -> int:
        return int(self.lib.dt_ctx_kernel_launches(self.h))

    def set_mem_limit(self, nbytes: int):
        """Caps the device memory this context's calls allocate (0: no cap);
        a call that would cross it raises DTError(DT_ERR_NOMEM)."""
        _lib.check(self.lib.dt_ctx_set_mem_limit(self.h, ctypes.c_uint64(int(nbytes))))

    def mem_usage(self):
        """(bytes held now, most bytes held since creation)."""
        a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        _lib.check(self.lib.dt_ctx_mem_usage(self.h, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def selftest_wait_timeout(self, limit_cycles: int):
        """Runs the bounded-wait self-test kernel; raises DTError(DT_ERR_TIMEOUT)
        when its wait ran out (it always does: nothing arrives on it)."""
        _lib.check(self.lib.dt_selftest_wait_timeout(self.h, ctypes.c_int64(int(limit_cycles))))

    # -- operators -----------------------------------------------------------
    def ttm(self, X, M, n: int):
        """Y = X x_n M (Function::ttm)."""
        self._bind(X, M)
        shape = list(X.shape)
        J = int(M.shape[0])
        xb, mb = _Buf(X), _Buf(M)
        out_shape = shape.copy()
        out_shape[n] = J
        Y = _alloc_like(xb.torch, out_shape, device=getattr(X, "device", None))
        yb = _Buf(Y)
        s = _shape_arr(shape)
        _lib.check(self.lib.dt_ttm_f64(self.h, xb.ptr, len(shape), _i64p(s), n, mb.ptr,
                                       J, yb.ptr))
        return Y

    def gram(self, X, n: int):
        self._bind(X)
        xb = _Buf(X)
        G = _alloc_like(xb.torch, [X.shape[n], X.shape[n]], device=getattr(X, "device", None))
        gb = _Buf(G)
        s = _shape_arr(X.shape)
        _lib.check(self.lib.dt_gram_f64(self.h, xb.ptr, X.ndim if not xb.torch else X.dim(),
                                        _i64p(s), n, gb.ptr))
        return G

    def gram_noalloc(self, X, n: int, G):
        """gram() into a caller-provided G, allocating nothing
        (dt_gram_f64_noalloc): X and G must be torch CUDA float64 tensors."""
        if not (_is_torch(X) and _is_torch(G) and X.is_cuda and G.is_cuda):
            raise TypeError("gram_noalloc needs torch CUDA tensors for X and G")
        self._bind(X, G)
        xb, gb = _Buf(X), _Buf(G)
        s = _shape_arr(X.shape)
        _lib.check(self.lib.dt_gram_f64_noalloc(self.h, xb.ptr, X.dim(), _i64p(s), n, gb.ptr))
        return G

    def ttt_except(self, A, B, n: int):
        self._bind(A, B)
        ab, bb = _Buf(A), _Buf(B)
        nd = len(A.shape)
        C = _alloc_like(ab.torch, [A.shape[n], B.shape[n]], device=getattr(A, "device", None))
        cb = _Buf(C)
        sa, sb = _shape_arr(A.shape), _shape_arr(B.shape)
        _lib.check(self.lib.dt_ttt_except_f64(self.h, ab.ptr, _i64p(sa), bb.ptr, _i64p(sb),
                                              nd, n, cb.ptr))
        return C

    def fnorm(self, X) -> float:
        self._bind(X)
        xb = _Buf(X)
        out = ctypes.c_double()
        n = int(np.prod(X.shape))
        _lib.check(self.lib.dt_fnorm_f64(self.h, xb.ptr, n, ctypes.byref(out)))
        return out.value

    def matmul(self, A, B, transA=False, transB=False):
        """C = op(A) op(B) (Operator::matmulNN/NT/TN)."""
        self._bind(A, B)
        A = np.asfortranarray(A, dtype=np.float64)
        B = np.asfortranarray(B, dtype=np.float64)
        m = A.shape[1] if transA else A.shape[0]
        k = A.shape[0] if transA else A.shape[1]
        n = B.shape[0] if transB else B.shape[1]
        C = np.zeros((m, n), order="F")
        _lib.check(self.lib.dt_matmul_f64(self.h, int(transA), int(transB), m, n, k,
                                          A.ctypes.data, B.ctypes.data, C.ctypes.data))
        return C

    def reduced_qr(self, A):
        self._bind(A)
        A = np.asfortranarray(A, dtype=np.float64)
        m, n = A.shape
        Q = np.zeros((m, n), order="F")
        R = np.zeros((n, n), order="F")
        _lib.check(self.lib.dt_reduced_qr_f64(self.h, A.ctypes.data, m, n, Q.ctypes.data,
                                              R.ctypes.data))
        return Q, R

    def inverse(self, A):
        self._bind(A)
        A = np.asfortranarray(A, dtype=np.float64)
        out = np.zeros_like(A, order="F")
        _lib.check(self.lib.dt_inverse_f64(self.h, A.ctypes.data, A.shape[0], out.ctypes.data))
        return out

    def orth2(self, A):
        """Row orthonormalisation of the R x I matrix A (Operator::orth2)."""
        self._bind(A)
        a = np.asfortranarray(np.array(A, dtype=np.float64, copy=True))
        _lib.check(self.lib.dt_orth2_f64(self.h, a.ctypes.data, a.shape[0], a.shape[1]))
        return a

    def als(self, Y, n, L0, iters=5):
        self._bind(Y)
        yb = _Buf(Y)
        L0 = np.asfortranarray(L0, dtype=np.float64)
        Q = np.zeros_like(L0, order="F")
        s = _shape_arr(Y.shape)
        _lib.check(self.lib.dt_als_f64(self.h, yb.ptr, len(Y.shape), _i64p(s), n,
                                       L0.ctypes.data, L0.shape[1], iters, Q.ctypes.data))
        return Q

    def ttm_tc(self, X, U, n: int, split: bool = False):
        """Y = X x_n U^T on the tensor cores (FP32 in/out, BF16 or hi+lo
        operands).  U is I_n x J."""
        self._bind(X, U)
        X = np.asfortranarray(X, dtype=np.float32)
        U = np.asfortranarray(U, dtype=np.float64)
        shape = list(X.shape)
        J = int(U.shape[1])
        out_shape = shape.copy()
        out_shape[n] = J
        Y = np.zeros(out_shape, dtype=np.float32, order="F")
        s = _shape_arr(shape)
        _lib.check(self.lib.dt_ttm_tc(self.h, X.ctypes.data, len(shape), _i64p(s), n,
                                      U.ctypes.data, J, int(split), Y.ctypes.data))
        return Y

    def gram_tc(self, Y, split: bool = False):
        """S = Y Y^T for a row-major I x K FP32 matrix, on the tensor cores."""
        self._bind(Y)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        I, K = Y.shape
        S = np.zeros((I, I), order="F")
        _lib.check(self.lib.dt_gram_tc(self.h, Y.ctypes.data, I, K, int(split), S.ctypes.data))
        return S

    # -- dense HOOI ----------------------------------------------------------
    def hooi_dense(self, X, ranks, *, init="randn", seed=1, U0=None, max_sweeps=5, tol=0.0,
                   inner_iters=5, precision=DT_PREC_FP64, refine_sweeps=0, verbose=False,
                   want_factors=True, want_core=True, profile=False, shape=None,
                   device_out=False):
        """Algorithm::Tucker::HOOI_ALS.  X: numpy or torch (float64/float32),
        column-major.  Returns (G, U, report-dict); with device_out and a CUDA
        torch X, G and U are float64 CUDA tensors with column-major strides,
        views of one device allocation (no copy back to the host), else numpy
        arrays."""
        self._bind(X)
        is_torch = _is_torch(X)
        if is_torch:
            import torch
            dtype = _lib.DT_F64 if X.dtype == torch.float64 else _lib.DT_F32
            xptr = ctypes.c_void_p(X.data_ptr())
            # A torch buffer holds the column-major data; pass the tensor
            # shape explicitly when the buffer is flat.
            shape = list(shape) if shape is not None else list(X.shape)
        else:
            X = np.asarray(X)
            if X.dtype not in (np.float64, np.float32):
                X = X.astype(np.float64)
            X = np.asfortranarray(X)
            dtype = _lib.DT_F64 if X.dtype == np.float64 else _lib.DT_F32
            xptr = ctypes.c_void_p(X.ctypes.data)
            shape = list(X.shape)
        N = len(shape)
        ranks = [int(r) for r in ranks]
        opts = HooiOpts()
        self.lib.dt_hooi_default_opts(ctypes.byref(opts))
        opts.init = {"randn": DT_INIT_RANDN_LIBC, "hosvd": DT_INIT_HOSVD,
                     "given": DT_INIT_GIVEN}[init if U0 is None else "given"]
        opts.seed = seed
        opts.max_sweeps = max_sweeps
        opts.tol = tol
        opts.inner_iters = inner_iters
        opts.precision = precision
        opts.refine_sweeps = refine_sweeps
        opts.verbose = int(verbose)
        opts.profile = int(profile)
        on_device = bool(device_out and is_torch and X.is_cuda)
        if on_device:
            import torch
            G, U = _column_major_outputs(shape, ranks, want_core,
                                         want_factors or U0 is not None, X.device)
            if U0 is not None:
                for n in range(N):
                    U[n].copy_(torch.as_tensor(np.asarray(U0[n], dtype=np.float64)))
            gptr = ctypes.c_void_p(G.data_ptr()) if G is not None else None
            Uptr = (ctypes.c_void_p * N)(*[u.data_ptr() for u in U]) if U is not None else None
        else:
            G = np.zeros(ranks, order="F") if want_core else None
            U = ([np.zeros((shape[n], ranks[n]), order="F") for n in range(N)]
                 if (want_factors or U0 is not None) else None)
            if U0 is not None:
                for n in range(N):
                    U[n][...] = np.asarray(U0[n], dtype=np.float64)
            gptr = ctypes.c_void_p(G.ctypes.data) if G is not None else None
            Uptr = (ctypes.c_void_p * N)(*[u.ctypes.data for u in U]) if U is not None else None
        rep = HooiReport()
        s, r = _shape_arr(shape), _shape_arr(ranks)
        _lib.check(self.lib.dt_hooi_dense(self.h, xptr, dtype, N, _i64p(s), _i64p(r),
                                          ctypes.byref(opts), gptr, Uptr, ctypes.byref(rep)))
        return G, U, rep.as_dict()

    # -- learned warm start ------------------------------------------------------
    def ws_loss_grad(self, U, E, D):
        """Autoencoder loss |D E U - U|^2 / N and its gradients (dt_ws_loss_grad).
        U: n x N, E: k x n, D: n x k (numpy, float64).  Returns (loss, gE, gD)."""
        self._bind()
        U = np.asfortranarray(U, dtype=np.float64)
        E = np.asfortranarray(E, dtype=np.float64)
        D = np.asfortranarray(D, dtype=np.float64)
        n, N = U.shape
        k = E.shape[0]
        loss = np.zeros(1)
        gE = np.zeros((k, n), order="F")
        gD = np.zeros((n, k), order="F")
        _lib.check(self.lib.dt_ws_loss_grad(self.h, U.ctypes.data, n, N, k, E.ctypes.data,
                                            D.ctypes.data, loss.ctypes.data, gE.ctypes.data,
                                            gD.ctypes.data))
        return float(loss[0]), gE, gD

    def ws_train(self, U, k, steps=400, lr=0.02, seed=1):
        """Trains the warm-start autoencoder on the columns of U (n x N).
        Returns (E, D, loss history)."""
        self._bind()
        U = np.asfortranarray(U, dtype=np.float64)
        n, N = U.shape
        E = np.zeros((k, n), order="F")
        D = np.zeros((n, k), order="F")
        hist = np.zeros(max(steps, 1))
        _lib.check(self.lib.dt_ws_train(self.h, U.ctypes.data, n, N, k, steps, lr, seed,
                                        E.ctypes.data, D.ctypes.data, hist.ctypes.data))
        return E, D, hist[:steps]

    def ws_init(self, X, ranks, D, shape=None, sketch_sweeps=0):
        """Warm-start factors for dense HOOI from decoder D (dt_ws_init).
        X: numpy or torch (float32/float64, column-major).  Returns
        (U list, fit of the sketch, fit of the initial factors)."""
        self._bind(X)
        if _is_torch(X):
            import torch
            dtype = _lib.DT_F64 if X.dtype == torch.float64 else _lib.DT_F32
            xptr = ctypes.c_void_p(X.data_ptr())
            shape = list(shape) if shape is not None else list(X.shape)
        else:
            X = np.asfortranarray(X)
            dtype = _lib.DT_F64 if X.dtype == np.float64 else _lib.DT_F32
            xptr = ctypes.c_void_p(X.ctypes.data)
            shape = list(X.shape)
        D = np.asfortranarray(D, dtype=np.float64)
        k = D.shape[1]
        N = len(shape)
        U = [np.zeros((shape[m], ranks[m]), order="F") for m in range(N)]
        Uptr = (ctypes.c_void_p * N)(*[u.ctypes.data for u in U])
        fs, fi = ctypes.c_double(), ctypes.c_double()
        s, r = _shape_arr(shape), _shape_arr(ranks)
        _lib.check(self.lib.dt_ws_init(self.h, xptr, dtype, N, _i64p(s), _i64p(r),
                                       D.ctypes.data, k, int(sketch_sweeps), Uptr,
                                       ctypes.byref(fs), ctypes.byref(fi)))
        return U, fs.value, fi.value

    # -- batched ---------------------------------------------------------------
    @staticmethod
    def pack_batched(tensors, ranks, U0=None):
        """Packs many small 3-way tensors for dt_hooi_batched: returns a dict
        with the concatenated FP32 data ``X``, the ``shapes``/``ranks``
        tables, the element offsets ``xoff``/``uoff``/``goff`` and (given
        U0, a list of 3-lists of initial factors) the packed FP64 ``U``."""
        count = len(tensors)
        shapes = np.array([t.shape for t in tensors], dtype=np.int64).reshape(-1)
        rk = np.array(ranks, dtype=np.int64).reshape(-1)
        sizes = [int(np.prod(t.shape)) for t in tensors]
        xoff = np.zeros(count, dtype=np.int64)
        xoff[1:] = np.cumsum(sizes)[:-1]
        X = np.empty(int(sum(sizes)), dtype=np.float32)
        for t, x in enumerate(tensors):
            X[xoff[t]:xoff[t] + sizes[t]] = np.asarray(x, dtype=np.float32).reshape(-1, order="F")
        usz = [int(tensors[t].shape[n]) * int(ranks[t][n]) for t in range(count) for n in range(3)]
        uoff = np.zeros(3 * count, dtype=np.int64)
        uoff[1:] = np.cumsum(usz)[:-1]
        gsz = [int(np.prod(r)) for r in ranks]
        goff = np.zeros(count, dtype=np.int64)
        goff[1:] = np.cumsum(gsz)[:-1]
        out = {"count": count, "shapes": shapes, "ranks": rk, "X": X, "xoff": xoff,
               "uoff": uoff, "goff": goff, "u_size": int(sum(usz)), "g_size": int(sum(gsz)),
               "shape_list": [tuple(int(v) for v in t.shape) for t in tensors],
               "rank_list": [tuple(int(v) for v in r) for r in ranks]}
        if U0 is not None:
            U = np.empty(out["u_size"])
            for t in range(count):
                for n in range(3):
                    o = uoff[3 * t + n]
                    U[o:o + usz[3 * t + n]] = np.asarray(U0[t][n], dtype=np.float64).reshape(
                        -1, order="F")
            out["U"] = U
        return out

    def hooi_batched_packed(self, packed, U, G, relerr, X=None, sweeps=10, inner_iters=5,
                            block_threads=0):
        """dt_hooi_batched on packed buffers (pack_batched): X (default
        packed["X"]), U (in/out), G and relerr (out) may be numpy arrays (host,
        staged by the library) or torch CUDA tensors (device-resident).
        Returns the report dict."""
        X = packed["X"] if X is None else X
        self._bind(X, U, G, relerr)
        xb = _Buf(X, dtype=np.float32, fortran=False)
        ub = _Buf(U, fortran=False)
        gb = _Buf(G, fortran=False)
        eb = _Buf(relerr, fortran=False)
        rep = _lib.BatchedReport()
        _lib.check(self.lib.dt_hooi_batched(
            self.h, packed["count"], _i64p(packed["shapes"]), _i64p(packed["ranks"]), xb.ptr,
            _i64p(packed["xoff"]), sweeps, inner_iters, ub.ptr, _i64p(packed["uoff"]), gb.ptr,
            _i64p(packed["goff"]), eb.ptr, block_threads, ctypes.byref(rep)))
        return rep.as_dict()

    def hooi_batched(self, tensors, ranks, U0, sweeps=10, inner_iters=5, block_threads=0):
        """HOOI of many small 3-way tensors in one launch (dt_hooi_batched).
        tensors: list of FP32 arrays; ranks: list of 3-tuples; U0: list of
        3-lists of initial factors.  Returns (U, G, relerr, report)."""
        pk = self.pack_batched(tensors, ranks, U0)
        U = pk["U"]
        G = np.zeros(pk["g_size"])
        relerr = np.zeros(pk["count"])
        report = self.hooi_batched_packed(pk, U, G, relerr, sweeps=sweeps,
                                          inner_iters=inner_iters, block_threads=block_threads)
        return (*self.unpack_batched(pk, U, G), relerr, report)

    @staticmethod
    def unpack_batched(packed, U, G):
        """Per-tensor factor lists and cores from packed U and G (host arrays)."""
        U = np.asarray(U)
        G = np.asarray(G)
        Uo, Go = [], []
        for t, (shape, r) in enumerate(zip(packed["shape_list"], packed["rank_list"])):
            fac = []
            for n in range(3):
                o = packed["uoff"][3 * t + n]
                fac.append(np.reshape(U[o:o + shape[n] * r[n]], (shape[n], r[n]), order="F"))
            Uo.append(fac)
            o = packed["goff"][t]
            Go.append(np.reshape(G[o:o + int(np.prod(r))], r, order="F"))
        return Uo, Go

    # -- Summary profiler --------------------------------------------------------
    def summary_enable(self, on: bool = True):
        """Summary::init / finalize: record named, nested device-timed ranges."""
        self._bind()
        _lib.check(self.lib.dt_summary_enable(self.h, int(on)))

    def summary_reset(self):
        _lib.check(self.lib.dt_summary_reset(self.h))

    def summary_table(self) -> str:
        """Summary::print_summary's table of the recorded ranges (recording
        restarts afterwards)."""
        need = ctypes.c_int64()
        buf = ctypes.create_string_buffer(1 << 22)
        _lib.check(self.lib.dt_summary_table(self.h, buf, len(buf), ctypes.byref(need)))
        return buf.value.decode()

    # -- sparse ----------------------------------------------------------------
    def sptensor(self, idx, vals, shape):
        return SpTensor(self, idx, vals, shape)

    def _tns_handle(self, path=None, data=None):
        self._bind()
        h, nd, nz = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int64()
        if path is not None:
            _lib.check(self.lib.dt_tns_read(self.h, os.fsencode(path), ctypes.byref(h),
                                            ctypes.byref(nd), ctypes.byref(nz)))
        else:
            buf = np.frombuffer(bytes(data), dtype=np.uint8)
            _lib.check(self.lib.dt_tns_parse(self.h, buf.ctypes.data, buf.size, ctypes.byref(h),
                                             ctypes.byref(nd), ctypes.byref(nz)))
        return h, nd.value, nz.value

    def read_tns(self, path=None, data=None):
        """read_data<double> on the device (dt_tns_read / dt_tns_parse): a .tns
        file by path, or its bytes.  Returns (idx: list of 0-based int64
        arrays, vals, dims)."""
        h, nd, nz = self._tns_handle(path, data)
        try:
            dims = np.zeros(nd, dtype=np.int64)
            idx = [np.zeros(nz, dtype=np.int64) for _ in range(nd)]
            vals = np.zeros(nz)
            ptrs = (ctypes.c_void_p * nd)(*[i.ctypes.data for i in idx])
            _lib.check(self.lib.dt_tns_copy(self.h, h, _i64p(dims), ptrs, vals.ctypes.data))
        finally:
            self.lib.dt_tns_destroy(h)
        return idx, vals, dims

    def sptensor_from_tns(self, path=None, data=None):
        """The parsed file as a device-built SpTensor (dt_tns_to_sptensor), with
        no host round trip of the nonzeros."""
        h, nd, nz = self._tns_handle(path, data)
        try:
            dims = np.zeros(nd, dtype=np.int64)
            _lib.check(self.lib.dt_tns_copy(self.h, h, _i64p(dims), None, None))
            sp = SpTensor.__new__(SpTensor)
            sp.ctx, sp.lib, sp.ndim, sp.nnz = self, self.lib, nd, nz
            sp.shape = [int(d) for d in dims]
            sh = ctypes.c_void_p()
            _lib.check(self.lib.dt_tns_to_sptensor(self.h, h, ctypes.byref(sh)))
            sp.h = sh
        finally:
            self.lib.dt_tns_destroy(h)
        return sp


class SpTensor:
    """Device-resident COO tensor with per-mode sorted copies (dt_sptensor)."""

    def __init__(self, ctx: Context, idx, vals, shape):
        self.ctx = ctx
        self.lib = ctx.lib
        ctx._bind()
        self.ndim = len(shape)
        self.shape = [int(s) for s in shape]
        idx = [np.ascontiguousarray(i, dtype=np.int64) for i in idx]
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.nnz = int(vals.shape[0])
        ptrs = (ctypes.c_void_p * self.ndim)(*[i.ctypes.data for i in idx])
        s = _shape_arr(self.shape)
        h = ctypes.c_void_p()
        _lib.check(self.lib.dt_sptensor_create(ctx.h, self.nnz, self.ndim, ptrs,
                                               vals.ctypes.data, _i64p(s), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.dt_sptensor_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _Ut(self, Ut):
        arrs = [np.ascontiguousarray(u, dtype=np.float64) for u in Ut]
        return arrs, (ctypes.c_void_p * self.ndim)(*[a.ctypes.data for a in arrs])

    def fnorm(self) -> float:
        out = ctypes.c_double()
        _lib.check(self.lib.dt_sp_fnorm(self.ctx.h, self.h, ctypes.byref(out)))
        return out.value

    @staticmethod
    def _kron_len(R, mode):
        P = 1
        for m, r in enumerate(R):
            if m != mode:
                P *= int(r)
        return P

    def ttmc_mTR(self, Ut, R, mode):
        keep, ptrs = self._Ut(Ut)
        r = _shape_arr(R)
        L = np.zeros((self._kron_len(R, mode), int(R[mode])), order="F")
        _lib.check(self.lib.dt_sp_ttmc_mTR(self.ctx.h, self.h, ptrs, _i64p(r), mode,
                                           L.ctypes.data))
        return L

    def ttmc_mTL(self, Ut, R, mode, L):
        keep, ptrs = self._Ut(Ut)
        r = _shape_arr(R)
        Lf = np.asfortranarray(L, dtype=np.float64)
        out = np.zeros((self.shape[mode], int(R[mode])))
        _lib.check(self.lib.dt_sp_ttmc_mTL(self.ctx.h, self.h, ptrs, _i64p(r), mode,
                                           Lf.ctypes.data, out.ctypes.data))
        return out

    def ttmc_rows(self, Ut, R, mode):
        keep, ptrs = self._Ut(Ut)
        r = _shape_arr(R)
        Y = np.zeros((self.shape[mode], self._kron_len(R, mode)))
        _lib.check(self.lib.dt_sp_ttmc_rows(self.ctx.h, self.h, ptrs, _i64p(r), mode,
                                            Y.ctypes.data))
        return Y

    def _dense_args(self, M, idx):
        """Factor pointers (J_m x I_m col-major, None for modes not in idx),
        row counts and the mode list for dt_sp_ttmc_dense_f64 / mettmc."""
        idx = [int(m) for m in idx]
        keep, ptrs = [], (ctypes.c_void_p * self.ndim)()
        J = np.zeros(self.ndim, dtype=np.int64)
        for m in range(self.ndim):
            if m in idx:
                a = np.asfortranarray(M[m], dtype=np.float64)
                if a.shape[1] != self.shape[m]:
                    raise ValueError(f"M[{m}] must be J x {self.shape[m]}")
                keep.append(a)
                ptrs[m] = a.ctypes.data
                J[m] = a.shape[0]
        ids = (ctypes.c_int * max(1, len(idx)))(*idx)
        out_shape = [int(J[m]) if m in idx else self.shape[m] for m in range(self.ndim)]
        return keep, ptrs, J, ids, out_shape

    def ttmc_dense(self, M, idx):
        """Function::ttmc(SpTensor, M, idx, ...): A x_{m in idx} M[m] as a dense
        column-major array (M[m] is J_m x I_m; modes outside idx keep I_m)."""
        keep, ptrs, J, ids, out_shape = self._dense_args(M, idx)
        Y = np.zeros(out_shape, order="F")
        _lib.check(self.lib.dt_sp_ttmc_dense_f64(self.ctx.h, self.h, ptrs, _i64p(J), ids,
                                                 len(list(idx)), Y.ctypes.data))
        return Y

    def mettmc(self, M, idx, level):
        """Function::mettmc: the same result, the `level` least-compressing
        modes (I_m / J_m) contracted densely after the sparse TTMc."""
        keep, ptrs, J, ids, out_shape = self._dense_args(M, idx)
        Y = np.zeros(out_shape, order="F")
        _lib.check(self.lib.dt_sp_mettmc_f64(self.ctx.h, self.h, ptrs, _i64p(J), ids,
                                             len(list(idx)), int(level), Y.ctypes.data))
        return Y

    def hooi(self, R, max_sweeps, Ut0):
        Ut = [np.ascontiguousarray(u, dtype=np.float64).copy() for u in Ut0]
        ptrs = (ctypes.c_void_p * self.ndim)(*[a.ctypes.data for a in Ut])
        r = _shape_arr(R)
        last = self.ndim - 1
        G = np.zeros((self._kron_len(R, last), int(R[last])), order="F")
        rep = HooiReport()
        _lib.check(self.lib.dt_sp_hooi(self.ctx.h, self.h, _i64p(r), max_sweeps, ptrs,
                                       G.ctypes.data, ctypes.byref(rep)))
        return G, Ut, rep.as_dict()
