"""ctypes access to the oracle (test infrastructure only).

``orc``  -- the CPU restatement in ``posit_oracle.c`` (``liborc.so``; built on demand
            with gcc if missing).
``ref``  -- the reference's own sources compiled here (``_ref/libposit_ref.so``), or
            ``None`` where it was not built (it needs the reference tree).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may use this package, and only as the checker / CPU baseline.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_c = ctypes


def _load_orc():
    path = os.path.join(HERE, "liborc.so")
    if not os.path.exists(path):
        from . import build_oracle
        build_oracle.build_oracle()
    lib = ctypes.CDLL(path)
    u32, i32, i64 = _c.c_uint32, _c.c_int, _c.c_int64
    for name in ("orc_p32_add", "orc_p32_sub", "orc_p32_mul", "orc_p32_div"):
        getattr(lib, name).argtypes = [u32, u32]
        getattr(lib, name).restype = u32
    for name in ("orc_p32_sqrt", "orc_p32_neg", "orc_p32_abs"):
        getattr(lib, name).argtypes = [u32]
        getattr(lib, name).restype = u32
    lib.orc_p32_from_double.argtypes = [_c.c_double]
    lib.orc_p32_from_double.restype = u32
    lib.orc_p32_to_double.argtypes = [u32]
    lib.orc_p32_to_double.restype = _c.c_double
    for name in ("orc_p32_add_n", "orc_p32_mul_n", "orc_p32_div_n"):
        getattr(lib, name).argtypes = [_U32P, _U32P, _U32P, i64]
    lib.orc_p32_sqrt_n.argtypes = [_U32P, _U32P, i64]
    lib.orc_p32_from_double_n.argtypes = [_F64P, _U32P, i64]
    lib.orc_p32_to_double_n.argtypes = [_U32P, _F64P, i64]
    gemm_args = [_c.c_char, _c.c_char, i32, i32, i32, u32, _U32P, i32, _U32P, i32, u32, _U32P, i32]
    lib.orc_rgemm.argtypes = gemm_args
    lib.orc_rgemm.restype = i32
    lib.orc_rgemm_cols.argtypes = gemm_args + [i32, i32]
    lib.orc_rgemm_cols.restype = i32
    lib.orc_num_threads.restype = i32
    lib.orc_iramax.argtypes = [i32, _U32P, i32]
    lib.orc_iramax.restype = i32
    lib.orc_rtrsm.argtypes = [_c.c_char] * 4 + [i32, i32, u32, _U32P, i32, _U32P, i32]
    lib.orc_rtrsm.restype = i32
    lib.orc_rsyrk.argtypes = [_c.c_char, _c.c_char, i32, i32, u32, _U32P, i32, u32, _U32P, i32]
    lib.orc_rsyrk.restype = i32
    lib.orc_rgemv.argtypes = [_c.c_char, i32, i32, u32, _U32P, i32, _U32P, i32, u32, _U32P, i32]
    lib.orc_rgemv.restype = i32
    lib.orc_rgetrf.argtypes = [i32, i32, _U32P, i32, _I32P, i32]
    lib.orc_rgetrf.restype = i32
    lib.orc_rgetrf2.argtypes = [i32, i32, _U32P, i32, _I32P]
    lib.orc_rgetrf2.restype = i32
    lib.orc_rgetrs.argtypes = [_c.c_char, i32, i32, _U32P, i32, _I32P, _U32P, i32]
    lib.orc_rgetrs.restype = i32
    lib.orc_rpotrf.argtypes = [_c.c_char, i32, _U32P, i32, i32]
    lib.orc_rpotrf.restype = i32
    lib.orc_rpotrf2.argtypes = [_c.c_char, i32, _U32P, i32]
    lib.orc_rpotrf2.restype = i32
    lib.orc_rpotrs.argtypes = [_c.c_char, i32, i32, _U32P, i32, _U32P, i32]
    lib.orc_rpotrs.restype = i32
    return lib


def _load_ref():
    path = os.path.join(HERE, "_ref", "libposit_ref.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    u32, i32, i64 = _c.c_uint32, _c.c_int, _c.c_int64
    lib.ref_p32_add.argtypes = [u32, u32]
    lib.ref_p32_add.restype = u32
    lib.ref_p32_mul.argtypes = [u32, u32]
    lib.ref_p32_mul.restype = u32
    lib.ref_p32_add_n.argtypes = [_U32P, _U32P, _U32P, i64]
    lib.ref_p32_mul_n.argtypes = [_U32P, _U32P, _U32P, i64]
    lib.ref_set_nb.argtypes = [i32]
    lib.ref_rgemm.argtypes = [_c.c_char, _c.c_char, i32, i32, i32, u32, _U32P, i32, _U32P, i32, u32, _U32P, i32]
    lib.ref_rsyrk.argtypes = [_c.c_char, _c.c_char, i32, i32, u32, _U32P, i32, u32, _U32P, i32]
    lib.ref_rtrsm.argtypes = [_c.c_char] * 4 + [i32, i32, u32, _U32P, i32, _U32P, i32]
    lib.ref_rgemv.argtypes = [_c.c_char, i32, i32, u32, _U32P, i32, _U32P, i32, u32, _U32P, i32]
    lib.ref_iramax.argtypes = [i32, _U32P, i32]
    lib.ref_iramax.restype = i32
    lib.ref_rgetrf.argtypes = [i32, i32, _U32P, i32, _I32P, i32]
    lib.ref_rgetrf.restype = i32
    lib.ref_rgetrs.argtypes = [_c.c_char, i32, i32, _U32P, i32, _I32P, _U32P, i32]
    lib.ref_rgetrs.restype = i32
    lib.ref_rpotrf.argtypes = [_c.c_char, i32, _U32P, i32, i32]
    lib.ref_rpotrf.restype = i32
    lib.ref_rpotrs.argtypes = [_c.c_char, i32, i32, _U32P, i32, _U32P, i32]
    lib.ref_rpotrs.restype = i32
    return lib


def load_ref_dropin():
    """The reference's own Rgetrf_opencl / Rpotrf_opencl linked against the B200 RgemmG
    (oracle/_ref/libposit_ref_dropin.so), or None where it was not built.  Loading it
    loads the CUDA library, so only GPU tests call this."""
    path = os.path.join(HERE, "_ref", "libposit_ref_dropin.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    i32 = _c.c_int
    lib.refd_rgetrf_opencl.argtypes = [i32, i32, _U32P, i32, _I32P, i32]
    lib.refd_rgetrf_opencl.restype = i32
    lib.refd_rpotrf_opencl.argtypes = [_c.c_char, i32, _U32P, i32, i32]
    lib.refd_rpotrf_opencl.restype = i32
    return lib


orc = _load_orc()
ref = _load_ref()

P32_ONE = 0x40000000
P32_NAR = 0x80000000
P32_MINUS_ONE = 0xC0000000


def from_double(x):
    """float64 array -> posit32 patterns (correctly rounded; unpinned vs SoftPosit)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(x.shape, dtype=np.uint32)
    orc.orc_p32_from_double_n(x.reshape(-1), out.reshape(-1), x.size)
    return out


def to_double(u):
    u = np.ascontiguousarray(u, dtype=np.uint32)
    out = np.empty(u.shape, dtype=np.float64)
    orc.orc_p32_to_double_n(u.reshape(-1), out.reshape(-1), u.size)
    return out


def p32(x):
    """One double -> posit32 pattern."""
    return int(orc.orc_p32_from_double(float(x)))


def rgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, cols=None):
    """Oracle Rgemm on flat column-major uint32 buffers; C updated in place.
    ``cols=(j0, j1)`` restricts the work to those columns of C."""
    args = (ta.encode(), tb.encode(), m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
    if cols is None:
        return orc.orc_rgemm(*args)
    return orc.orc_rgemm_cols(*args, cols[0], cols[1])


def rgemm_cols_checked(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, j0, j1):
    """Columns j0..j1-1 of the Rgemm result, computed by the reference's own compiled
    Rgemm (``ref``) where it was built, else by the restatement: returns a copy of those
    columns of C (ldc x (j1 - j0), flat) after the update, and which checker ran.

    Columns of C are independent in every order of Rgemm.cpp:163-247, so the reference
    routine runs on the slice: op(B)'s columns j0..j1-1 start at B[j0*ldb] ('N') or at
    B[j0] ('T'/'C', B is n x k), and C's at C[j0*ldc]."""
    A = np.ascontiguousarray(A, dtype=np.uint32)
    B = np.ascontiguousarray(B, dtype=np.uint32)
    Cs = np.array(C[j0 * ldc:j1 * ldc], dtype=np.uint32, copy=True)
    w = j1 - j0
    if ref is not None:
        Bs = B[j0 * ldb:] if tb in "nN" else B[j0:]
        ref.ref_rgemm(ta.encode(), tb.encode(), m, w, k, alpha, A, lda, np.ascontiguousarray(Bs), ldb,
                      beta, Cs, ldc)
        return Cs, "reference"
    Cf = np.array(C, dtype=np.uint32, copy=True)
    rc = orc.orc_rgemm_cols(ta.encode(), tb.encode(), m, n, k, alpha, A, lda, B, ldb, beta, Cf, ldc, j0, j1)
    if rc != 0:
        raise ValueError(f"oracle Rgemm info {rc}")
    return Cf[j0 * ldc:j1 * ldc].copy(), "port"
