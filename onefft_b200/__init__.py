"""onefft_b200 — OneFFT's power-of-two FP32 complex FFT as hand-written sm_100a CUDA.

The product is ``libonefft_cuda.so`` with the C ABI of ``include/onefft.h`` (OneFFT's own API)
and ``include/onefft_cuda.h`` (device-pointer, batched and uneven-batch additions). This module
is the Python host mirror of that interface, shaped like OneFFT's C++ layer
(include/onefft.h:123-169 of OneFFT): ``forward``/``inverse`` without plan management, a
``Plan`` that owns the tables of one size, ``cache_prepare``/``cache_clear`` and
``implementation``. Errors follow OneFFT's contract: an invalid size raises ``ValueError`` (the C
call returned -1 / NULL) and leaves any output buffer untouched.

There is no CPU fallback: if the CUDA library is missing, importing the entry points raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libonefft_cuda.so")

_c_float_p = ctypes.POINTER(ctypes.c_float)
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p

# exported symbols of the C ABI, in header order (include/onefft.h, include/onefft_cuda.h)
C_SYMBOLS = (
    "onefft_forward", "onefft_inverse", "onefft_cache_prepare", "onefft_cache_clear",
    "onefft_plan_create", "onefft_plan_destroy", "onefft_plan_forward", "onefft_plan_inverse",
    "onefft_plan_size", "onefft_implementation",
    "onefft_dev_forward_batched", "onefft_dev_inverse_batched", "onefft_dev_adjoint_batched",
    "onefft_dev_forward_weighted", "onefft_dev_inverse_weighted",
    "onefft_dev_weighted_power_loss",
    "onefft_plan_forward_batched", "onefft_plan_inverse_batched",
    "onefft_plan_create_split", "onefft_plan_create_tiles", "onefft_plan_create_bf16x3", "onefft_plan_create_bf16x6",
    "onefft_plan_passes",
    "onefft_uneven_create", "onefft_uneven_create_split", "onefft_uneven_destroy", "onefft_uneven_span", "onefft_uneven_execute",
    "onefft_uneven_status",
    "onefft_uneven_execute_noalloc",
    "onefft_columns_create", "onefft_columns_destroy", "onefft_columns_execute", "onefft_columns_status",
    "onefft_last_error", "onefft_plan_status", "onefft_debug_fail_alloc", "onefft_debug_twiddles",
    "onefft_debug_launch_count", "onefft_debug_expire_waits",
)

_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library with typed entry points (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built: run `python -m onefft_b200.build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.onefft_forward.argtypes = [_vp, _vp, _sz]
    L.onefft_forward.restype = ctypes.c_int
    L.onefft_inverse.argtypes = [_vp, _vp, _sz]
    L.onefft_inverse.restype = ctypes.c_int
    L.onefft_cache_prepare.argtypes = [_sz]
    L.onefft_cache_prepare.restype = ctypes.c_int
    L.onefft_cache_clear.argtypes = []
    L.onefft_cache_clear.restype = None
    L.onefft_plan_create.argtypes = [_sz]
    L.onefft_plan_create.restype = _vp
    L.onefft_plan_create_split.argtypes = [_sz, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.onefft_plan_create_split.restype = _vp
    L.onefft_plan_create_tiles.argtypes = [_sz, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int]
    L.onefft_plan_create_tiles.restype = _vp
    L.onefft_plan_create_bf16x3.argtypes = [_sz, ctypes.c_int]
    L.onefft_plan_create_bf16x3.restype = _vp
    L.onefft_plan_create_bf16x6.argtypes = [_sz, ctypes.c_int]
    L.onefft_plan_create_bf16x6.restype = _vp
    L.onefft_plan_destroy.argtypes = [_vp]
    L.onefft_plan_destroy.restype = None
    L.onefft_plan_forward.argtypes = [_vp, _vp, _vp]
    L.onefft_plan_forward.restype = None
    L.onefft_plan_inverse.argtypes = [_vp, _vp, _vp]
    L.onefft_plan_inverse.restype = None
    L.onefft_plan_size.argtypes = [_vp]
    L.onefft_plan_size.restype = _sz
    L.onefft_plan_passes.argtypes = [_vp, ctypes.POINTER(ctypes.c_int)]
    L.onefft_plan_passes.restype = ctypes.c_int
    L.onefft_implementation.argtypes = []
    L.onefft_implementation.restype = ctypes.c_char_p
    for name in ("onefft_dev_forward_batched", "onefft_dev_inverse_batched", "onefft_dev_adjoint_batched"):
        f = getattr(L, name)
        f.argtypes = [_vp, _vp, _vp, _sz, _vp]
        f.restype = ctypes.c_int
    for name in ("onefft_dev_forward_weighted", "onefft_dev_inverse_weighted"):
        f = getattr(L, name)
        f.argtypes = [_vp, _vp, _vp, _sz, _vp, _vp, _vp]
        f.restype = ctypes.c_int
    L.onefft_dev_weighted_power_loss.argtypes = [_vp, _vp, _vp, _vp, _sz, _vp, _vp]
    L.onefft_dev_weighted_power_loss.restype = ctypes.c_int
    for name in ("onefft_plan_forward_batched", "onefft_plan_inverse_batched"):
        f = getattr(L, name)
        f.argtypes = [_vp, _vp, _vp, _sz]
        f.restype = ctypes.c_int
    L.onefft_uneven_create.argtypes = [_vp, _sz]
    L.onefft_uneven_create.restype = _vp
    L.onefft_uneven_create_split.argtypes = [_vp, _sz, ctypes.POINTER(ctypes.c_int)]
    L.onefft_uneven_create_split.restype = _vp
    L.onefft_uneven_destroy.argtypes = [_vp]
    L.onefft_uneven_destroy.restype = None
    L.onefft_uneven_span.argtypes = [_vp]
    L.onefft_uneven_span.restype = _sz
    L.onefft_uneven_execute.argtypes = [_vp, _vp, _vp, _vp]
    L.onefft_uneven_execute.restype = ctypes.c_int
    L.onefft_uneven_status.argtypes = [_vp]
    L.onefft_uneven_status.restype = ctypes.c_int
    L.onefft_uneven_execute_noalloc.argtypes = [_vp, _sz, _vp, _vp, _vp]
    L.onefft_uneven_execute_noalloc.restype = ctypes.c_int
    L.onefft_columns_create.argtypes = [_sz, _sz, _sz, ctypes.c_ulonglong, ctypes.c_ulonglong]
    L.onefft_columns_create.restype = _vp
    L.onefft_columns_destroy.argtypes = [_vp]
    L.onefft_columns_destroy.restype = None
    L.onefft_columns_execute.argtypes = [_vp, _vp, _vp, ctypes.c_int, _vp]
    L.onefft_columns_execute.restype = ctypes.c_int
    L.onefft_columns_status.argtypes = [_vp]
    L.onefft_columns_status.restype = ctypes.c_int
    L.onefft_last_error.argtypes = []
    L.onefft_last_error.restype = ctypes.c_char_p
    L.onefft_debug_fail_alloc.argtypes = [ctypes.c_int]
    L.onefft_debug_fail_alloc.restype = None
    L.onefft_debug_twiddles.argtypes = [ctypes.c_uint, _sz, _vp]
    L.onefft_debug_twiddles.restype = ctypes.c_int
    L.onefft_debug_launch_count.argtypes = []
    L.onefft_debug_launch_count.restype = ctypes.c_ulonglong
    L.onefft_plan_status.argtypes = [_vp]
    L.onefft_plan_status.restype = ctypes.c_int
    L.onefft_debug_expire_waits.argtypes = [ctypes.c_int]
    L.onefft_debug_expire_waits.restype = ctypes.c_int
    _lib = L
    return L


def implementation() -> str:
    return lib().onefft_implementation().decode()


def last_error() -> str:
    return lib().onefft_last_error().decode()


def _as_interleaved(x) -> np.ndarray:
    """A C-contiguous float32 view (2n floats) of complex64 or interleaved float32 data."""
    a = np.asarray(x)
    if a.dtype == np.complex64:
        a = a.view(np.float32)
    if a.dtype != np.float32:
        raise TypeError("expected complex64 or interleaved float32 data")
    if not a.flags.c_contiguous:
        a = np.ascontiguousarray(a)
    return a.reshape(-1)


def _out_like(a: np.ndarray, out):
    if out is None:
        return np.empty_like(a)
    o = _as_interleaved(out)
    if o.size != a.size:
        raise ValueError("output size differs from input size")
    return o


def forward(x, out=None):
    """OneFFT's onefft_forward on host data (complex64 or interleaved float32)."""
    a = _as_interleaved(x)
    o = _out_like(a, out)
    if lib().onefft_forward(a.ctypes.data, o.ctypes.data, a.size // 2) != 0:
        raise ValueError(f"onefft_forward failed: {last_error()}")
    return o


def inverse(x, out=None):
    """OneFFT's onefft_inverse on host data (unnormalised)."""
    a = _as_interleaved(x)
    o = _out_like(a, out)
    if lib().onefft_inverse(a.ctypes.data, o.ctypes.data, a.size // 2) != 0:
        raise ValueError(f"onefft_inverse failed: {last_error()}")
    return o


def cache_prepare(n: int) -> None:
    if lib().onefft_cache_prepare(n) != 0:
        raise ValueError(f"onefft_cache_prepare({n}) failed: {last_error()}")


def cache_clear() -> None:
    lib().onefft_cache_clear()


class Plan:
    """Owns the device tables of one size (OneFFT's onefft::Plan, include/onefft.h:136-167)."""

    def __init__(self, n: int, split: tuple[int, ...] | None = None, cols: tuple[int, ...] | None = None,
                 l2_keep: bool = True, chunk: int = 0, bf16x3: bool = False, require_accepted: bool = False,
                 tma: bool = False, fuse_lag: int = 0, bf16x6: bool = False):
        """split: log2 pass lengths (None = tuned table); cols: log2 tile widths per pass;
        chunk: three passes only, log2 last-digit columns per L2-resident chunk (0 = none);
        fuse_lag: with chunk and tma, run passes 0 and 1 as one persistent kernel with pass 1
        trailing pass 0 by this many chunks (ONEFFT_OPT_FUSED; 0 = separate launches);
        bf16x3 / bf16x6: the split-BF16 tensor-core variant of three (hi/lo) or six
        (hi/mid/lo) product terms (require_accepted: only at sizes where it meets the FP32 error
        bound)."""
        L = lib()
        if bf16x3 or bf16x6:
            f = L.onefft_plan_create_bf16x6 if bf16x6 else L.onefft_plan_create_bf16x3
            h = f(n, int(require_accepted))
        elif split is None:
            h = L.onefft_plan_create(n)
        else:
            arr = (ctypes.c_int * len(split))(*split)
            carr = (ctypes.c_int * len(split))(*cols) if cols is not None else None
            # ONEFFT_OPT_L2_KEEP | ONEFFT_OPT_TMA | ONEFFT_OPT_FUSED | ONEFFT_OPT_LAG(fuse_lag)
            options = (1 if l2_keep else 0) | (2 if tma else 0) | ((4 | (fuse_lag << 8)) if fuse_lag else 0)
            h = L.onefft_plan_create_tiles(n, len(split), arr, carr, options, int(chunk))
        if not h:
            raise ValueError(f"no plan for n={n}: {last_error()}")
        self._h = h
        self.n = int(n)

    @property
    def handle(self) -> int:
        if not self._h:
            raise ValueError("plan was destroyed")
        return self._h

    def size(self) -> int:
        return int(lib().onefft_plan_size(self.handle))

    def passes(self) -> tuple[int, ...]:
        buf = (ctypes.c_int * 3)()
        k = lib().onefft_plan_passes(self.handle, buf)
        return tuple(buf[i] for i in range(k))

    def status(self) -> int:
        """onefft_plan_status: 0, or the error code of a kernel failure recorded since the last
        call (reading clears it); call after synchronising the streams the plan ran on."""
        return int(lib().onefft_plan_status(self.handle))

    def check(self) -> None:
        """Raises if a kernel of this plan recorded a failure (see status())."""
        rc = self.status()
        if rc != 0:
            raise RuntimeError(f"transform failed on the device ({rc}): {last_error()}")

    def destroy(self) -> None:
        if getattr(self, "_h", None):
            lib().onefft_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def _host(self, x, out, inverse: bool, batch: int | None):
        a = _as_interleaved(x)
        o = _out_like(a, out)
        if batch is None:
            if a.size != 2 * self.n:
                raise ValueError("input size differs from the plan size")
            f = lib().onefft_plan_inverse if inverse else lib().onefft_plan_forward
            f(self.handle, a.ctypes.data, o.ctypes.data)
            err = last_error()
            if err:
                raise RuntimeError(err)
        else:
            if a.size != 2 * self.n * batch:
                raise ValueError("input size differs from batch * plan size")
            f = lib().onefft_plan_inverse_batched if inverse else lib().onefft_plan_forward_batched
            rc = f(self.handle, a.ctypes.data, o.ctypes.data, batch)
            if rc != 0:
                raise RuntimeError(f"batched transform failed ({rc}): {last_error()}")
        return o

    def forward(self, x, out=None, batch: int | None = None):
        return self._host(x, out, False, batch)

    def inverse(self, x, out=None, batch: int | None = None):
        return self._host(x, out, True, batch)

    # ---- device pointers (raw addresses; see onefft_b200.torch_ops for tensors) ----

    def dev_forward(self, d_in: int, d_out: int, batch: int = 1, stream: int = 0) -> None:
        rc = lib().onefft_dev_forward_batched(self.handle, d_in, d_out, batch, stream)
        if rc != 0:
            raise RuntimeError(f"onefft_dev_forward_batched failed ({rc}): {last_error()}")

    def dev_inverse(self, d_in: int, d_out: int, batch: int = 1, stream: int = 0) -> None:
        rc = lib().onefft_dev_inverse_batched(self.handle, d_in, d_out, batch, stream)
        if rc != 0:
            raise RuntimeError(f"onefft_dev_inverse_batched failed ({rc}): {last_error()}")

    def dev_weighted(self, d_in: int, d_out: int, batch: int = 1, pre: int | None = None, post: int | None = None,
                     inverse: bool = False, stream: int = 0) -> None:
        """out_b = post * T(pre * in_b) with the weights applied inside the transform kernels
        (onefft_dev_forward_weighted / _inverse_weighted); pre / post are device pointers to n
        complex values or None."""
        f = lib().onefft_dev_inverse_weighted if inverse else lib().onefft_dev_forward_weighted
        rc = f(self.handle, d_in, d_out, batch, pre, post, stream)
        if rc != 0:
            raise RuntimeError(f"onefft_dev_{'inverse' if inverse else 'forward'}_weighted failed ({rc}): {last_error()}")

    def dev_adjoint(self, d_grad_out: int, d_grad_in: int, batch: int = 1, stream: int = 0) -> None:
        rc = lib().onefft_dev_adjoint_batched(self.handle, d_grad_out, d_grad_in, batch, stream)
        if rc != 0:
            raise RuntimeError(f"onefft_dev_adjoint_batched failed ({rc}): {last_error()}")


DESC_DTYPE = np.dtype([("log2n", np.int32), ("inverse", np.int32), ("offset", np.int64)])


class UnevenBatch:
    """Many transforms of different power-of-two sizes run by one persistent launch
    (onefft_uneven_* in include/onefft_cuda.h). `desc` is a structured array of DESC_DTYPE, or
    three sequences (log2n, inverse, offset)."""

    def __init__(self, log2n, inverse=None, offset=None, split: dict[int, int] | None = None):
        """split: {log2 n: choice} for sizes 2^13 .. 2^16 (onefft_uneven_create_split; sizes not
        named take choice 0); None = the tuned choices (onefft_uneven_create)."""
        if inverse is None:
            d = np.ascontiguousarray(log2n, DESC_DTYPE)
        else:
            d = np.empty(len(log2n), DESC_DTYPE)
            d["log2n"], d["inverse"], d["offset"] = log2n, inverse, offset
        self.desc = d
        if split is None:
            h = lib().onefft_uneven_create(d.ctypes.data, d.size)
        else:
            choice = (ctypes.c_int * 17)(*[int(split.get(m, 0)) for m in range(17)])
            h = lib().onefft_uneven_create_split(d.ctypes.data, d.size, choice)
        if not h:
            raise ValueError(f"invalid uneven batch: {last_error()}")
        self._h = h

    @property
    def span(self) -> int:
        return int(lib().onefft_uneven_span(self._h))

    def execute(self, d_in: int, d_out: int, stream: int = 0) -> None:
        rc = lib().onefft_uneven_execute(self._h, d_in, d_out, stream)
        if rc != 0:
            raise RuntimeError(f"onefft_uneven_execute failed ({rc}): {last_error()}")

    def status(self) -> int:
        """onefft_uneven_status: 0, or the error code of a failed wait since the last call."""
        return int(lib().onefft_uneven_status(self._h))

    def destroy(self) -> None:
        if getattr(self, "_h", None):
            lib().onefft_uneven_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


SWAP_IN, SWAP_OUT = 1, 2  # ONEFFT_SWAP_IN / ONEFFT_SWAP_OUT


class Columns:
    """Transforms down the columns of a row-major n x cols matrix, written row-wise in `blocks`
    blocks, optionally times the four-step twiddle w_big_n^((col0 + b) k) of a larger transform
    (onefft_columns_* in include/onefft_cuda.h): out[((k / r) cols + b) r + k mod r] = Y_b[k],
    r = n / blocks."""

    def __init__(self, n: int, cols: int, blocks: int = 1, big_n: int = 0, col0: int = 0):
        h = lib().onefft_columns_create(n, cols, blocks, big_n, col0)
        if not h:
            raise ValueError(f"no column transform for n={n}, cols={cols}, blocks={blocks}, big_n={big_n}, "
                             f"col0={col0}: {last_error()}")
        self._h = h
        self.n, self.cols, self.blocks, self.big_n, self.col0 = int(n), int(cols), int(blocks), int(big_n), int(col0)

    def execute(self, d_in: int, d_out: int, flags: int = 0, stream: int = 0) -> None:
        """Enqueues the transform of n * cols complex values at d_in into d_out (device pointers;
        flags: SWAP_IN | SWAP_OUT)."""
        if not self._h:
            raise ValueError("column transform was destroyed")
        rc = lib().onefft_columns_execute(self._h, d_in, d_out, flags, stream)
        if rc != 0:
            raise RuntimeError(f"onefft_columns_execute failed ({rc}): {last_error()}")

    def status(self) -> int:
        """onefft_columns_status: 0, or the error code of a tile copy whose bounded wait ran out
        since the last call (reading clears it); call after synchronising the stream."""
        return int(lib().onefft_columns_status(self._h))

    def check(self) -> None:
        """Raises if a kernel of this column transform recorded a failure (see status())."""
        rc = self.status()
        if rc != 0:
            raise RuntimeError(f"column transform failed on the device ({rc}): {last_error()}")

    def destroy(self) -> None:
        if getattr(self, "_h", None):
            lib().onefft_columns_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


__all__ = ["forward", "inverse", "cache_prepare", "cache_clear", "Plan", "UnevenBatch", "DESC_DTYPE", "Columns",
           "SWAP_IN", "SWAP_OUT", "implementation", "last_error", "lib", "LIB_PATH", "C_SYMBOLS"]
