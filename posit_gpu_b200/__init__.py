"""posit_gpu_b200 -- bit-exact posit32 BLAS on B200 (sm_100a).

Host-side mirror of the reference's GPU GEMM interface (libRpack/mpblas_posit.h:49-55,
libRpack/def.h:63):

    initOpenCL()                      -> init()
    RgemmG(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
                                      -> Rgemm / RgemmG (host numpy buffers, synchronous)
    (device-resident form)            -> Rgemm_dev (torch CUDA tensors, stream-ordered)

posit32 values are their raw 32-bit patterns: ``alpha``/``beta`` are ints, matrices are
flat column-major ``numpy.uint32`` arrays (or any buffer of 4-byte elements) indexed as
``A[i + j*lda]``.  Errors are raised, never turned into a CPU fallback: an illegal
argument raises ``ValueError`` carrying the BLAS info code the reference's Mxerbla
would print, a CUDA failure raises ``RuntimeError``, and a missing library raises
``ImportError`` at import time.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libposit_gpu_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python posit_gpu_b200/build.py` "
        "(there is no CPU fallback)")

_lib = ctypes.CDLL(LIB_PATH)
_c = ctypes
_VP = _c.c_void_p
_GEMM_HEAD = [_c.c_char, _c.c_char, _c.c_int, _c.c_int, _c.c_int, _c.c_uint32, _VP, _c.c_int,
              _VP, _c.c_int, _c.c_uint32, _VP, _c.c_int]
_lib.posit_init.restype = _c.c_int
_lib.posit_rgemm.argtypes = _GEMM_HEAD
_lib.posit_rgemm.restype = _c.c_int
_lib.posit_rgemm_dev.argtypes = _GEMM_HEAD + [_VP, _c.c_size_t, _VP]
_lib.posit_rgemm_dev.restype = _c.c_int
_lib.posit_rgemm_dev_noalloc.argtypes = _GEMM_HEAD + [_VP]
_lib.posit_rgemm_dev_noalloc.restype = _c.c_int
_lib.posit_rgemm_workspace_size.argtypes = [_c.c_char, _c.c_char, _c.c_int, _c.c_int, _c.c_int]
_lib.posit_rgemm_workspace_size.restype = _c.c_size_t
_lib.posit_device_error.argtypes = [_c.c_int]
_lib.posit_device_error.restype = _c.c_int
_lib.posit_last_cuda_error.restype = _c.c_int
_lib.posit_profile_enable.argtypes = [_c.c_int]
_lib.posit_profile_read.argtypes = [_c.POINTER(_c.c_double), _c.POINTER(_c.c_longlong),
                                    _c.POINTER(_c.c_longlong), _c.c_int]
_lib.posit_from_double_dev.argtypes = [_VP, _VP, _c.c_size_t, _VP]
_lib.posit_from_double_dev.restype = _c.c_int
_lib.posit_to_double_dev.argtypes = [_VP, _VP, _c.c_size_t, _VP]
_lib.posit_to_double_dev.restype = _c.c_int
_I = _c.c_int
_lib.posit_rgetrf_dev.argtypes = [_I, _I, _VP, _I, _VP, _I, _VP, _VP]
_lib.posit_rgetrf.argtypes = [_I, _I, _VP, _I, _VP, _I, _c.POINTER(_I)]
_lib.posit_rgetrs_dev.argtypes = [_c.c_char, _I, _I, _VP, _I, _VP, _VP, _I, _VP]
_lib.posit_rgetrs.argtypes = [_c.c_char, _I, _I, _VP, _I, _VP, _VP, _I]
_lib.posit_rpotrf_dev.argtypes = [_c.c_char, _I, _VP, _I, _I, _VP, _VP]
_lib.posit_rpotrf.argtypes = [_c.c_char, _I, _VP, _I, _I, _c.POINTER(_I)]
_lib.posit_rpotrs_dev.argtypes = [_c.c_char, _I, _I, _VP, _I, _VP, _I, _VP]
_lib.posit_rpotrs.argtypes = [_c.c_char, _I, _I, _VP, _I, _VP, _I]
for _f in ("posit_rgetrf_dev", "posit_rgetrf", "posit_rgetrs_dev", "posit_rgetrs", "posit_rpotrf_dev",
           "posit_rpotrf", "posit_rpotrs_dev", "posit_rpotrs"):
    getattr(_lib, _f).restype = _I
_lib.posit_strerror.argtypes = [_c.c_int]
_lib.posit_strerror.restype = _c.c_char_p

P32_ZERO = 0x00000000
P32_ONE = 0x40000000
P32_MINUS_ONE = 0xC0000000
P32_NAR = 0x80000000


class PositError(RuntimeError):
    pass


def _check(rc, name):
    if rc == 0:
        return
    if rc > 0:
        # Mxerbla.cpp:70-73 prints this and exits; here it is an exception
        raise ValueError(f" ** On entry to {name} parameter number {rc:2d} had an illegal value")
    msg = _lib.posit_strerror(rc).decode()
    raise PositError(f"{name}: {msg} (code {rc}, cuda error {_lib.posit_last_cuda_error()})")


def _char(c):
    if isinstance(c, (bytes, bytearray)):
        c = c.decode()
    return str(c)[:1].encode() or b" "


def _host_ptr(x):
    if isinstance(x, np.ndarray):
        if x.dtype.itemsize != 4:
            raise TypeError("posit32 buffers hold 4-byte elements")
        if not x.flags.c_contiguous and not x.flags.f_contiguous:
            raise TypeError("buffer must be contiguous")
        return x.ctypes.data
    raise TypeError("host buffers must be numpy arrays of 4-byte elements")


def init():
    """Select the current device and create its context (replaces initOpenCL)."""
    _check(_lib.posit_init(), "init")


initOpenCL = init


def Rgemm(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """C <- alpha*op(A)*op(B) + beta*C on host buffers, bit-identical to the CPU Rgemm
    (libRpack/Rgemm.cpp:62-251) for every transpose case.  Synchronous; C in place."""
    _check(_lib.posit_rgemm(_char(transa), _char(transb), m, n, k, int(alpha) & 0xFFFFFFFF,
                            _host_ptr(A), lda, _host_ptr(B), ldb, int(beta) & 0xFFFFFFFF,
                            _host_ptr(C), ldc), "Rgemm ")


RgemmG = Rgemm


def workspace_size(transa, transb, m, n, k):
    return int(_lib.posit_rgemm_workspace_size(_char(transa), _char(transb), m, n, k))


def Rgemm_dev(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace=None,
              stream=None):
    """Device-resident Rgemm: A, B, C (and the optional workspace) are CUDA tensors of a
    4-byte dtype (raw posit patterns); enqueued on ``stream`` (default: torch's current
    stream); returns without synchronising."""
    import torch

    for t in (A, B, C):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.element_size() == 4):
            raise TypeError("Rgemm_dev takes CUDA tensors of 4-byte elements")
    if stream is None:
        stream = torch.cuda.current_stream(C.device)
    ws_ptr, ws_bytes = None, 0
    if workspace is not None:
        ws_ptr, ws_bytes = workspace.data_ptr(), workspace.numel() * workspace.element_size()
    _check(_lib.posit_rgemm_dev(_char(transa), _char(transb), m, n, k, int(alpha) & 0xFFFFFFFF,
                                A.data_ptr(), lda, B.data_ptr(), ldb, int(beta) & 0xFFFFFFFF,
                                C.data_ptr(), ldc, ws_ptr, ws_bytes, stream.cuda_stream), "Rgemm ")


def from_double_dev(x, out=None, stream=None):
    """float64 CUDA tensor -> posit32 patterns (int32 CUDA tensor), correctly rounded."""
    import torch
    if not (x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()):
        raise TypeError("from_double_dev takes a contiguous float64 CUDA tensor")
    if out is None:
        out = torch.empty(x.shape, dtype=torch.int32, device=x.device)
    stream = stream or torch.cuda.current_stream(x.device)
    _check(_lib.posit_from_double_dev(x.data_ptr(), out.data_ptr(), x.numel(), stream.cuda_stream),
           "from_double")
    return out


def to_double_dev(u, out=None, stream=None):
    """posit32 patterns (4-byte CUDA tensor) -> float64 CUDA tensor (exact)."""
    import torch
    if not (u.is_cuda and u.element_size() == 4 and u.is_contiguous()):
        raise TypeError("to_double_dev takes a contiguous 4-byte CUDA tensor")
    if out is None:
        out = torch.empty(u.shape, dtype=torch.float64, device=u.device)
    stream = stream or torch.cuda.current_stream(u.device)
    _check(_lib.posit_to_double_dev(u.data_ptr(), out.data_ptr(), u.numel(), stream.cuda_stream),
           "to_double")
    return out


# ---------------------------------------------------------------------------
# LAPACK (libRpack/mplapack_posit.h:38-52): LU and Cholesky, bit-identical to the CPU
# routines.  Host forms take numpy buffers (4-byte elements; ipiv int32) and return the
# reference's `info`; _dev forms take torch CUDA tensors and leave info on the device.
# ---------------------------------------------------------------------------
def _host_i32(x):
    if not (isinstance(x, np.ndarray) and x.dtype == np.int32):
        raise TypeError("ipiv must be a numpy int32 array")
    return x.ctypes.data


def Rgetrf(m, n, A, lda, ipiv, nb=0):
    """LU with partial pivoting in place (Rgetrf.cpp:32-137); ipiv 1-based. Returns info."""
    info = _I(0)
    _check(_lib.posit_rgetrf(m, n, _host_ptr(A), lda, _host_i32(ipiv), nb, _c.byref(info)), "Rgetrf")
    return info.value


def Rgetrs(trans, n, nrhs, A, lda, ipiv, B, ldb):
    """Solve with an Rgetrf factorization (Rgetrs.cpp:32-118), B overwritten."""
    _check(_lib.posit_rgetrs(_char(trans), n, nrhs, _host_ptr(A), lda, _host_i32(ipiv), _host_ptr(B), ldb),
           "Rgetrs")


def Rpotrf(uplo, n, A, lda, nb=0):
    """Cholesky in place (Rpotrf.cpp:32-154). Returns info."""
    info = _I(0)
    _check(_lib.posit_rpotrf(_char(uplo), n, _host_ptr(A), lda, nb, _c.byref(info)), "Rpotrf")
    return info.value


def Rpotrs(uplo, n, nrhs, A, lda, B, ldb):
    """Solve with an Rpotrf factor (Rpotrs.cpp:32-110), B overwritten."""
    _check(_lib.posit_rpotrs(_char(uplo), n, nrhs, _host_ptr(A), lda, _host_ptr(B), ldb), "Rpotrs")


def _stream_of(t, stream):
    import torch
    return (stream or torch.cuda.current_stream(t.device)).cuda_stream


def Rgetrf_dev(m, n, A, lda, ipiv, info, nb=0, stream=None):
    """Device LU: A (4-byte CUDA tensor), ipiv (int32 CUDA tensor, >= min(m,n)), info
    (int32 CUDA tensor, 1 element, written on the device).  Asynchronous."""
    _check(_lib.posit_rgetrf_dev(m, n, A.data_ptr(), lda, ipiv.data_ptr(), nb, info.data_ptr(),
                                 _stream_of(A, stream)), "Rgetrf")


def Rgetrs_dev(trans, n, nrhs, A, lda, ipiv, B, ldb, stream=None):
    _check(_lib.posit_rgetrs_dev(_char(trans), n, nrhs, A.data_ptr(), lda, ipiv.data_ptr(), B.data_ptr(), ldb,
                                 _stream_of(A, stream)), "Rgetrs")


def Rpotrf_dev(uplo, n, A, lda, info, nb=0, stream=None):
    _check(_lib.posit_rpotrf_dev(_char(uplo), n, A.data_ptr(), lda, nb, info.data_ptr(), _stream_of(A, stream)),
           "Rpotrf")


def Rpotrs_dev(uplo, n, nrhs, A, lda, B, ldb, stream=None):
    _check(_lib.posit_rpotrs_dev(_char(uplo), n, nrhs, A.data_ptr(), lda, B.data_ptr(), ldb,
                                 _stream_of(A, stream)), "Rpotrs")


# ---------------------------------------------------------------------------
# Batched factor-and-solve: one persistent launch, captured in a CUDA graph
# ---------------------------------------------------------------------------
BATCH_LU = 0
BATCH_CHOLESKY = 1
BATCH_MAX_N = 4096


class _BatchProblem(_c.Structure):
    _fields_ = [("kind", _c.c_int), ("n", _c.c_int), ("lda", _c.c_int), ("nrhs", _c.c_int), ("ldb", _c.c_int),
                ("A", _VP), ("B", _VP), ("ipiv", _VP), ("info", _VP)]


_lib.posit_batch_plan_create.argtypes = [_c.POINTER(_BatchProblem), _c.c_int, _c.POINTER(_VP)]
_lib.posit_batch_plan_create.restype = _c.c_int
_lib.posit_batch_plan_launch.argtypes = [_VP, _VP]
_lib.posit_batch_plan_launch.restype = _c.c_int
_lib.posit_batch_plan_destroy.argtypes = [_VP]


class BatchPlan:
    """Factor-and-solve many problems in one graph-captured persistent launch.

    problems: iterable of (kind, A, B, ipiv, info) with kind BATCH_LU / BATCH_CHOLESKY,
    A an n x n column-major CUDA tensor of 4-byte posit patterns (flat or 2-D), B its
    n x nrhs right-hand sides (flat, column-major), ipiv an int32 CUDA tensor of n
    entries (LU; may be None for Cholesky), info an int32 CUDA tensor of one entry.
    The tensors must stay alive while the plan is used."""

    def __init__(self, problems):
        probs = list(problems)
        arr = (_BatchProblem * max(1, len(probs)))()
        self._keep = []
        for i, (kind, A, B, ipiv, info) in enumerate(probs):
            n = int(round(A.numel() ** 0.5))
            if n * n != A.numel():
                raise ValueError("A must be square")
            nrhs = B.numel() // n if n else 0
            arr[i] = _BatchProblem(kind, n, max(1, n), nrhs, max(1, n), A.data_ptr(), B.data_ptr(),
                                   ipiv.data_ptr() if ipiv is not None else None, info.data_ptr())
            self._keep.append((A, B, ipiv, info))
        h = _VP()
        _check(_lib.posit_batch_plan_create(arr, len(probs), _c.byref(h)), "batch plan")
        self._h = h

    def launch(self, stream=None):
        import torch
        st = stream or torch.cuda.current_stream()
        _check(_lib.posit_batch_plan_launch(self._h, st.cuda_stream), "batch launch")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.posit_batch_plan_destroy(h)
            self._h = None


class _BatchGemm(_c.Structure):
    _fields_ = [("transa", _c.c_char), ("transb", _c.c_char), ("m", _c.c_int), ("n", _c.c_int), ("k", _c.c_int),
                ("alpha", _c.c_uint32), ("beta", _c.c_uint32), ("A", _VP), ("lda", _c.c_int), ("B", _VP),
                ("ldb", _c.c_int), ("C", _VP), ("ldc", _c.c_int)]


_lib.posit_batch_gemm_plan_create.argtypes = [_c.POINTER(_BatchGemm), _c.c_int, _c.POINTER(_c.c_int),
                                              _c.POINTER(_VP), _c.POINTER(_c.c_int)]
_lib.posit_batch_gemm_plan_create.restype = _c.c_int


class BatchGemmPlan(BatchPlan):
    """Many independent Rgemm calls in one graph-captured persistent launch.

    problems: iterable of (transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
    with A, B, C CUDA tensors of 4-byte posit patterns (kept alive by the plan).
    tile_table: 9 ints (size bucket -> tile shape), default: the built-in table."""

    def __init__(self, problems, tile_table=None):
        probs = list(problems)
        arr = (_BatchGemm * max(1, len(probs)))()
        self._keep = []
        for i, (ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc) in enumerate(probs):
            arr[i] = _BatchGemm(_char(ta), _char(tb), m, n, k, int(alpha) & 0xFFFFFFFF, int(beta) & 0xFFFFFFFF,
                                A.data_ptr(), lda, B.data_ptr(), ldb, C.data_ptr(), ldc)
            self._keep.append((A, B, C))
        tt = None
        if tile_table is not None:
            tt = (_c.c_int * 9)(*[int(x) for x in tile_table])
        h, bad = _VP(), _c.c_int(-1)
        rc = _lib.posit_batch_gemm_plan_create(arr, len(probs), tt, _c.byref(h), _c.byref(bad))
        if rc > 0:
            raise ValueError(f" ** On entry to Rgemm  parameter number {rc:2d} had an illegal value "
                             f"(batch problem {bad.value})")
        _check(rc, "batch gemm plan")
        self._h = h


NOALLOC_SCRATCH_BYTES = 64 << 20
POSIT_E_NOALLOC_LIMIT = -6


def Rgemm_dev_noalloc(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream=None):
    """Rgemm_dev for callers that cannot allocate device memory: the scratch is a
    static 64 MiB device array inside the library (shared by all calls on a device; calls
    that overlap on the GPU race).  Shapes needing more scratch raise PositError."""
    import torch

    for t in (A, B, C):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.element_size() == 4):
            raise TypeError("Rgemm_dev_noalloc takes CUDA tensors of 4-byte elements")
    if stream is None:
        stream = torch.cuda.current_stream(C.device)
    _check(_lib.posit_rgemm_dev_noalloc(_char(transa), _char(transb), m, n, k, int(alpha) & 0xFFFFFFFF,
                                        A.data_ptr(), lda, B.data_ptr(), ldb, int(beta) & 0xFFFFFFFF,
                                        C.data_ptr(), ldc, stream.cuda_stream), "Rgemm ")


def device_error(clear=True):
    return int(_lib.posit_device_error(1 if clear else 0))


def profile_enable(on=True):
    """Record CUDA events around every GEMM main-kernel launch (on its stream)."""
    _lib.posit_profile_enable(1 if on else 0)


def profile_read(reset=True):
    """-> (main-kernel milliseconds, main-kernel launches, all kernel launches)."""
    ms, mains, alls = _c.c_double(), _c.c_longlong(), _c.c_longlong()
    _lib.posit_profile_read(_c.byref(ms), _c.byref(mains), _c.byref(alls), 1 if reset else 0)
    return ms.value, mains.value, alls.value


# ---------------------------------------------------------------------------
# Served solves (no reference counterpart): include/posit_gpu.h, posit_server_*
# ---------------------------------------------------------------------------
class _ServerConfig(_c.Structure):
    _fields_ = [("memory_budget", _c.c_size_t), ("max_inflight", _c.c_int), ("max_queue", _c.c_int),
                ("lanes", _c.c_int), ("launch_threads", _c.c_int), ("batch_max_n", _c.c_int), ("nb", _c.c_int),
                ("cache_off", _c.c_int), ("batch_lanes", _c.c_int), ("order_window_ms", _c.c_int),
                ("priority_n", _c.c_int)]


class _SolveRequest(_c.Structure):
    _fields_ = [("kind", _c.c_int), ("n", _c.c_int), ("nrhs", _c.c_int), ("matrix_id", _c.c_longlong),
                ("A", _VP), ("B", _VP), ("X", _VP)]


class _SolveResult(_c.Structure):
    _fields_ = [("status", _c.c_int), ("info", _c.c_int), ("cache_hit", _c.c_int), ("path", _c.c_int),
                ("queue_ms", _c.c_double), ("latency_ms", _c.c_double)]


class _ServerStats(_c.Structure):
    _fields_ = [(f, _c.c_longlong) for f in ("submitted", "completed", "failed", "cancelled", "cache_hits",
                                            "cache_misses", "evictions", "batched_units", "blocked_units",
                                            "inflight_peak")] + \
               [(f, _c.c_size_t) for f in ("budget_bytes", "bytes_in_use", "bytes_peak", "cached_bytes")]


_lib.posit_server_create.argtypes = [_c.POINTER(_ServerConfig), _c.POINTER(_VP)]
_lib.posit_server_submit.argtypes = [_VP, _c.POINTER(_SolveRequest), _c.POINTER(_c.c_longlong)]
_lib.posit_server_wait.argtypes = [_VP, _c.c_longlong, _c.POINTER(_SolveResult)]
_lib.posit_server_poll.argtypes = [_VP, _c.c_longlong, _c.POINTER(_SolveResult)]
_lib.posit_server_cancel.argtypes = [_VP, _c.c_longlong]
_lib.posit_server_get_stats.argtypes = [_VP, _c.POINTER(_ServerStats)]
_lib.posit_server_destroy.argtypes = [_VP]
for _f in ("posit_server_create", "posit_server_submit", "posit_server_wait", "posit_server_poll",
           "posit_server_cancel", "posit_server_get_stats"):
    getattr(_lib, _f).restype = _I

SOLVE_LU = BATCH_LU
SOLVE_CHOLESKY = BATCH_CHOLESKY
E_QUEUE_FULL, E_CANCELLED, E_NOT_CACHED, E_MISMATCH, E_UNKNOWN_TICKET = -8, -9, -10, -11, -12


def _buf_ptr(x):
    """Host buffer of 4-byte posit patterns: a numpy array or a CPU torch tensor
    (page-locked ones are copied asynchronously)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return _host_ptr(x)
    if getattr(x, "is_cuda", False) or not hasattr(x, "data_ptr"):
        raise TypeError("served requests take host buffers (numpy arrays or CPU tensors)")
    if x.element_size() != 4 or not x.is_contiguous():
        raise TypeError("posit32 buffers hold 4-byte elements, contiguous")
    return x.data_ptr()


class Server:
    """Served Ax = b solves: continuous admission under a device-memory budget, batched
    small problems, blocked large ones overlapping on the GPU, and an on-device factor
    cache keyed by matrix id.  Every solution is bit-identical to the per-call path.

        srv = Server(memory_budget=150e9)
        t = srv.submit(SOLVE_LU, n, nrhs, A, B, X, matrix_id=7)   # host buffers
        res = srv.wait(t)     # {'status', 'info', 'cache_hit', 'path', 'queue_ms', 'latency_ms'}
    """

    def __init__(self, memory_budget=0, max_inflight=0, max_queue=0, lanes=0, launch_threads=0,
                 batch_max_n=0, nb=0, cache=True, batch_lanes=0, order_window_ms=0, priority_n=0):
        cfg = _ServerConfig(int(memory_budget), max_inflight, max_queue, lanes, launch_threads, batch_max_n, nb,
                            0 if cache else 1, batch_lanes, order_window_ms, priority_n)
        h = _VP()
        _check(_lib.posit_server_create(_c.byref(cfg), _c.byref(h)), "server")
        self._h = h
        self._keep = {}

    def submit(self, kind, n, nrhs, A, B, X, matrix_id=-1):
        """Queue one request (host buffers, column-major, lda = ldb = n); returns a ticket.
        A may be None when matrix_id names a cached factor."""
        q = _SolveRequest(kind, n, nrhs, matrix_id, _buf_ptr(A), _buf_ptr(B), _buf_ptr(X))
        t = _c.c_longlong()
        _check(_lib.posit_server_submit(self._h, _c.byref(q), _c.byref(t)), "server submit")
        self._keep[t.value] = (A, B, X)
        return t.value

    @staticmethod
    def _result(r):
        return {"status": r.status, "info": r.info, "cache_hit": bool(r.cache_hit), "path": r.path,
                "queue_ms": r.queue_ms, "latency_ms": r.latency_ms}

    def wait(self, ticket):
        r = _SolveResult()
        _check(_lib.posit_server_wait(self._h, ticket, _c.byref(r)), "server wait")
        self._keep.pop(ticket, None)
        return self._result(r)

    def poll(self, ticket):
        """The result if the request is finished, else None."""
        r = _SolveResult()
        rc = _lib.posit_server_poll(self._h, ticket, _c.byref(r))
        if rc < 0:
            _check(rc, "server poll")
        if rc == 0:
            return None
        self._keep.pop(ticket, None)
        return self._result(r)

    def cancel(self, ticket):
        """True if the request was cancelled before admission."""
        rc = _lib.posit_server_cancel(self._h, ticket)
        if rc < 0:
            _check(rc, "server cancel")
        return rc == 0

    def stats(self):
        st = _ServerStats()
        _check(_lib.posit_server_get_stats(self._h, _c.byref(st)), "server stats")
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.posit_server_destroy(h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
