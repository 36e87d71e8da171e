"""CPU oracle for the onefft_b200 tests — test infrastructure, not part of the product.

Python access (ctypes + numpy) to:

* ``liboracle.so`` — the plain-C restatement of OneFFT's transform (twiddle rule of
  src/onefft.c:115-141, portable radix-2 path of src/onefft.c:158-230), the FP64 checks of the
  reference's tests (tests/test_onefft.c:31-71, 99-101, 142-164), the seeded generators and the
  threaded CPU timing harness over the restatement;
* ``_ref/libonefft_ref.so`` / ``_ref/libonefft_ref_portable.so`` — the reference library
  compiled from its unmodified sources (SIMD build and its ONEFFT_NO_SIMD portable build), each
  with the same timing harness.

Only tests, the smoke check and the benchmark's CPU-baseline leg import this package. The
product (``onefft_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libonefft_ref.so")
REF_PORTABLE_SO = os.path.join(HERE, "_ref", "libonefft_ref_portable.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_sz = ctypes.c_size_t


# Where the OneFFT tree is mounted on the machine that builds the checker (read-only; the GPU
# machines have no copy and use the prebuilt oracle/_ref/). ONEFFT_REFERENCE_DIR overrides it.
REFERENCE_DIR = os.environ.get("ONEFFT_REFERENCE_DIR", "/root/reference")


def build(reference_dir: str | None = None) -> None:
    """Compile liboracle.so and, when the reference sources exist, oracle/_ref/ from them."""
    env = dict(os.environ)
    args = ["make", "-C", HERE, "--no-print-directory"]
    ref = reference_dir or REFERENCE_DIR
    if ref and os.path.exists(os.path.join(ref, "src", "onefft.c")):
        args.append(f"REF={ref}")
    subprocess.run(args, check=True, env=env, stdout=subprocess.DEVNULL)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class _Lib:
    _cache: dict[str, ctypes.CDLL] = {}

    @classmethod
    def get(cls, path: str) -> ctypes.CDLL:
        if path not in cls._cache:
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} is not built (run oracle.build())")
            lib = ctypes.CDLL(path)
            lib.cpu_bench_batched.restype = ctypes.c_double
            lib.cpu_bench_batched.argtypes = [_sz, _sz, ctypes.c_int, ctypes.c_int, _f32p, _f32p, ctypes.c_int]
            lib.cpu_bench_uneven.restype = ctypes.c_double
            lib.cpu_bench_uneven.argtypes = [_i32p, _i64p, _i32p, _sz, ctypes.c_int, _f32p, _f32p, ctypes.c_int]
            lib.cpu_bench_impl.restype = ctypes.c_char_p
            lib.cpu_bench_ncores.restype = ctypes.c_int
            cls._cache[path] = lib
        return cls._cache[path]


def lib() -> ctypes.CDLL:
    L = _Lib.get(ORACLE_SO)
    if not getattr(L, "_typed", False):
        L.oracle_root_f64.argtypes = [ctypes.c_uint64, ctypes.c_uint, _f64p, _f64p]
        L.oracle_twiddle_table.argtypes = [ctypes.c_uint, _sz, _f32p]
        L.oracle_fft_f32.argtypes = [_f32p, _f32p, _sz, ctypes.c_int]
        L.oracle_fft_f32.restype = ctypes.c_int
        L.oracle_fft_f64.argtypes = [_f64p, _sz, ctypes.c_int]
        L.oracle_fft_f64_from_f32.argtypes = [_f32p, _f64p, _sz, ctypes.c_int]
        L.oracle_dft_bins.argtypes = [_f32p, _sz, ctypes.c_int, _u64p, _sz, _f64p]
        L.oracle_rel_rms.argtypes = [_f32p, _f64p, _sz]
        L.oracle_rel_rms.restype = ctypes.c_double
        L.oracle_max_abs.argtypes = [_f32p, _f64p, _sz]
        L.oracle_max_abs.restype = ctypes.c_double
        L.oracle_tolerance.argtypes = [ctypes.c_uint]
        L.oracle_tolerance.restype = ctypes.c_double
        L.oracle_gen_uniform.argtypes = [ctypes.POINTER(ctypes.c_uint32), _f32p, _sz]
        L.oracle_gen_normal.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _f32p, _sz]
        L.oracle_gen_wide.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _f32p, _sz]
        L.oracle_plan_create.restype = ctypes.c_void_p
        L.oracle_plan_create.argtypes = [_sz]
        L.oracle_plan_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_plan_forward.argtypes = [ctypes.c_void_p, _f32p, _f32p]
        L.oracle_plan_inverse.argtypes = [ctypes.c_void_p, _f32p, _f32p]
        L._typed = True
    return L


def reference_lib(portable: bool = False) -> ctypes.CDLL:
    """The reference library built from its own sources, typed for its public C API."""
    L = _Lib.get(REF_PORTABLE_SO if portable else REF_SO)
    if not getattr(L, "_typed", False):
        L.onefft_forward.argtypes = [_f32p, _f32p, _sz]
        L.onefft_forward.restype = ctypes.c_int
        L.onefft_inverse.argtypes = [_f32p, _f32p, _sz]
        L.onefft_inverse.restype = ctypes.c_int
        L.onefft_plan_create.argtypes = [_sz]
        L.onefft_plan_create.restype = ctypes.c_void_p
        L.onefft_plan_destroy.argtypes = [ctypes.c_void_p]
        L.onefft_plan_forward.argtypes = [ctypes.c_void_p, _f32p, _f32p]
        L.onefft_plan_inverse.argtypes = [ctypes.c_void_p, _f32p, _f32p]
        L.onefft_implementation.restype = ctypes.c_char_p
        L._typed = True
    return L


def have_reference() -> bool:
    return os.path.exists(REF_SO)


# ---- generators -----------------------------------------------------------------------------

SEED_TESTS = 0x9E3779B9  # tests/test_onefft.c:57
SEED_BENCH = 0x12345678  # bench/bench.c:94


def gen_uniform(count_floats: int, state: int = SEED_TESTS) -> tuple[np.ndarray, int]:
    """xorshift32 uniform [-1,1) floats; returns (values, next state)."""
    out = np.empty(count_floats, np.float32)
    s = ctypes.c_uint32(state)
    lib().oracle_gen_uniform(ctypes.byref(s), _ptr(out, _f32p), count_floats)
    return out, s.value


def gen_normal(count_floats: int, seed: int, first: int = 0) -> np.ndarray:
    out = np.empty(count_floats, np.float32)
    lib().oracle_gen_normal(seed, first, _ptr(out, _f32p), count_floats)
    return out


def gen_wide(n_complex: int, seed: int, first_complex: int = 0) -> np.ndarray:
    out = np.empty(2 * n_complex, np.float32)
    lib().oracle_gen_wide(seed, first_complex, _ptr(out, _f32p), n_complex)
    return out


# ---- transforms and checks ------------------------------------------------------------------


def port_fft(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """The restated portable FP32 transform of interleaved floats x (2n)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    rc = lib().oracle_fft_f32(_ptr(x, _f32p), _ptr(out, _f32p), x.size // 2, int(inverse))
    if rc:
        raise ValueError("invalid size")
    return out


def ref_fft(x: np.ndarray, inverse: bool = False, portable: bool = False) -> np.ndarray:
    """The reference library's onefft_forward / onefft_inverse on interleaved floats x (2n)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    L = reference_lib(portable)
    f = L.onefft_inverse if inverse else L.onefft_forward
    if f(_ptr(x, _f32p), _ptr(out, _f32p), x.size // 2):
        raise ValueError("invalid size")
    return out


def ref_fft_batched(x: np.ndarray, n: int, inverse: bool = False) -> np.ndarray:
    """Reference transforms of every length-n slice of x (2n floats each), one shared plan."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    L = reference_lib()
    plan = L.onefft_plan_create(n)
    f = L.onefft_plan_inverse if inverse else L.onefft_plan_forward
    base_in, base_out = x.ctypes.data, out.ctypes.data
    for b in range(x.size // (2 * n)):
        f(plan, ctypes.cast(base_in + 8 * n * b, _f32p), ctypes.cast(base_out + 8 * n * b, _f32p))
    L.onefft_plan_destroy(plan)
    return out


def fft64(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """FP64 radix-2 FFT of FP32 interleaved x, as interleaved doubles (tests/test_onefft.c:31-55)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty(x.size, np.float64)
    lib().oracle_fft_f64_from_f32(_ptr(x, _f32p), _ptr(out, _f64p), x.size // 2, int(inverse))
    return out


def fft64_numpy(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """Second opinion: numpy's FP64 FFT (unnormalised in both directions), interleaved."""
    z = x.astype(np.float64).view(np.complex128)
    y = np.fft.ifft(z) * z.size if inverse else np.fft.fft(z)
    return np.ascontiguousarray(y).view(np.float64)


def columns_fp64(x: np.ndarray, n: int, cols: int, blocks: int = 1, big_n: int = 0, col0: int = 0,
                 flags: int = 0) -> np.ndarray:
    """FP64 statement of the column transform's contract (onefft_columns_execute,
    include/onefft_cuda.h): transforms down the columns of the n x cols matrix x (complex),
    times w_big_n^((col0 + b) k), out[((k / r) cols + b) r + k mod r] = Y_b[k], r = n / blocks;
    flags 1 / 2 exchange re/im of the input / of the result. Returns complex128. The exponent is
    reduced modulo big_n in integers before the angle is formed."""
    a = np.asarray(x).astype(np.complex128).reshape(n, cols)
    if flags & 1:
        a = a.imag + 1j * a.real
    y = np.fft.fft(a, axis=0)
    if big_n:
        t = ((col0 + np.arange(cols, dtype=np.int64))[None, :] * np.arange(n, dtype=np.int64)[:, None]) % big_n
        y = y * np.exp(-2j * np.pi * (t.astype(np.float64) / big_n))
    if flags & 2:
        y = y.imag + 1j * y.real
    r = n // blocks
    return np.ascontiguousarray(y.T.reshape(cols, blocks, r).transpose(1, 0, 2)).reshape(-1)


def dft_bins(x: np.ndarray, bins, inverse: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    b = np.ascontiguousarray(np.asarray(bins, np.uint64))
    out = np.empty(2 * b.size, np.float64)
    lib().oracle_dft_bins(_ptr(x, _f32p), x.size // 2, int(inverse), _ptr(b, _u64p), b.size, _ptr(out, _f64p))
    return out


def rel_rms(got: np.ndarray, want: np.ndarray) -> float:
    got = np.ascontiguousarray(got, np.float32).ravel()
    want = np.ascontiguousarray(want, np.float64).ravel()
    return lib().oracle_rel_rms(_ptr(got, _f32p), _ptr(want, _f64p), got.size)


def max_abs(got: np.ndarray, want: np.ndarray) -> float:
    got = np.ascontiguousarray(got, np.float32).ravel()
    want = np.ascontiguousarray(want, np.float64).ravel()
    return lib().oracle_max_abs(_ptr(got, _f32p), _ptr(want, _f64p), got.size // 2)


def tolerance(log2n: int) -> float:
    return 4e-7 + 1e-7 * log2n


def twiddle_table(log2n: int, count: int) -> np.ndarray:
    out = np.empty(2 * count, np.float32)
    lib().oracle_twiddle_table(log2n, count, _ptr(out, _f32p))
    return out


def root_f64(k: int, log2size: int) -> tuple[float, float]:
    re, im = ctypes.c_double(), ctypes.c_double()
    lib().oracle_root_f64(k, log2size, ctypes.byref(re), ctypes.byref(im))
    return re.value, im.value


# ---- CPU timing harness ---------------------------------------------------------------------


def cpu_bench_batched(n: int, batch: int, threads: int, inverse: bool, x: np.ndarray, out: np.ndarray,
                      samples: int = 3, kind: str = "reference") -> float:
    L = _Lib.get(REF_SO if kind == "reference" else ORACLE_SO)
    return L.cpu_bench_batched(n, batch, threads, int(inverse), _ptr(x, _f32p), _ptr(out, _f32p), samples)


def cpu_bench_uneven(log2n: np.ndarray, offset: np.ndarray, inverse: np.ndarray, threads: int, x: np.ndarray,
                     out: np.ndarray, samples: int = 3, kind: str = "reference") -> float:
    L = _Lib.get(REF_SO if kind == "reference" else ORACLE_SO)
    return L.cpu_bench_uneven(_ptr(log2n, _i32p), _ptr(offset, _i64p), _ptr(inverse, _i32p), log2n.size, threads,
                              _ptr(x, _f32p), _ptr(out, _f32p), samples)


def cpu_impl(kind: str = "reference") -> str:
    L = _Lib.get(REF_SO if kind == "reference" else ORACLE_SO)
    return L.cpu_bench_impl().decode()


def cpu_cores(kind: str = "reference") -> int:
    L = _Lib.get(REF_SO if kind == "reference" else ORACLE_SO)
    return int(L.cpu_bench_ncores())
