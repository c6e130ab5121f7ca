"""The product C-ABI library loads, exports every entry point include/posit_gpu.h
declares, and checks arguments with the reference's info codes (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(posit_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import posit_gpu_b200 as pg
    lib = ctypes.CDLL(pg.LIB_PATH)
    names = _declared()
    assert "posit_rgemm" in names and "posit_rgemm_dev" in names
    for nm in names:
        assert hasattr(lib, nm), nm


@pytest.mark.parametrize("args,info", [
    (("X", "N", 2, 2, 2, 2, 2, 2), 1),
    (("N", "Q", 2, 2, 2, 2, 2, 2), 2),
    (("N", "N", -1, 2, 2, 2, 2, 2), 3),
    (("N", "N", 2, -1, 2, 2, 2, 2), 4),
    (("N", "N", 2, 2, -1, 2, 2, 2), 5),
    (("N", "N", 4, 2, 2, 3, 2, 4), 8),
    (("T", "N", 2, 2, 4, 3, 4, 2), 8),
    (("N", "N", 2, 2, 4, 2, 3, 2), 10),
    (("N", "T", 2, 5, 2, 2, 4, 2), 10),
    (("N", "N", 5, 2, 2, 5, 2, 4), 13),
])
def test_argument_checks_return_rgemm_info(args, info):
    """Rgemm.cpp:107-128 order of checks; no CUDA call is made for a bad argument."""
    import posit_gpu_b200 as pg
    ta, tb, m, n, k, lda, ldb, ldc = args
    buf = np.zeros(64, dtype=np.uint32)
    rc = pg._lib.posit_rgemm(ta.encode(), tb.encode(), m, n, k, 0x40000000, buf.ctypes.data, lda,
                             buf.ctypes.data, ldb, 0, buf.ctypes.data, ldc)
    assert rc == info
    with pytest.raises(ValueError, match=f"parameter number {info:2d}"):
        pg.Rgemm(ta, tb, m, n, k, 0x40000000, buf, lda, buf, ldb, 0, buf, ldc)


def test_quick_returns_need_no_device():
    """m == 0, n == 0, or (alpha == 0 or k == 0) with beta == 1 return before any
    device work (Rgemm.cpp:134-136), leaving C untouched."""
    import posit_gpu_b200 as pg
    C = np.arange(16, dtype=np.uint32)
    before = C.copy()
    for (m, n, k, alpha, beta) in ((0, 4, 4, 1, 5), (4, 0, 4, 1, 5), (4, 4, 4, 0, 0x40000000),
                                   (4, 4, 0, 0x40000000, 0x40000000)):
        pg.Rgemm("N", "N", m, n, k, alpha, C, 4, C, 4, beta, C, 4)
    assert np.array_equal(C, before)


def test_lower_case_and_C_are_transposes():
    import posit_gpu_b200 as pg
    buf = np.zeros(64, dtype=np.uint32)
    for t in ("n", "t", "c", "C", "T"):
        rc = pg._lib.posit_rgemm(t.encode(), b"n", 0, 2, 2, 0, buf.ctypes.data, 2, buf.ctypes.data, 2, 0,
                                 buf.ctypes.data, 2)
        assert rc == 0


def test_strerror_and_workspace_size():
    import posit_gpu_b200 as pg
    assert pg._lib.posit_strerror(0) == b"success"
    assert b"argument" in pg._lib.posit_strerror(8)
    assert pg.workspace_size("N", "N", 0, 5, 5) == 0
    ws = pg.workspace_size("N", "T", 100, 70, 33)
    # decoded operands: 8 bytes per element of op(A) and op(B), padded to whole tiles,
    # plus one NaR flag byte per padded row and column
    assert ws >= 8 * (100 + 70) * 33 + 100 + 70
    assert ws < 8 * (100 + 70 + 2 * 64) * (33 + 16) + 1024
    assert pg.workspace_size("N", "T", 100, 70, 66) > ws


def test_server_needs_a_device_and_reports_it():
    """Without a GPU the request loop is not started: creation returns POSIT_E_NO_DEVICE
    and no thread or allocation is left behind."""
    import torch

    import posit_gpu_b200 as pg
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pg.PositError, match="no usable CUDA device"):
        pg.Server()
    for code, text in ((pg.E_QUEUE_FULL, b"queue"), (pg.E_CANCELLED, b"cancelled"),
                       (pg.E_NOT_CACHED, b"cached"), (pg.E_MISMATCH, b"matrix id"),
                       (pg.E_UNKNOWN_TICKET, b"ticket")):
        assert text in pg._lib.posit_strerror(code)


def test_built_in_panel_widths_match_the_tuning_table():
    """The widths nb <= 0 selects (compiled into the library) are the autotuner's table
    committed beside it (posit_gpu_b200/tuning_b200.json), for every tuned size and the
    sizes between."""
    import json
    import posit_gpu_b200 as pg
    lib = ctypes.CDLL(pg.LIB_PATH)
    lib.posit_tuned_panel_width.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.posit_tuned_panel_width.restype = ctypes.c_int
    table = json.load(open(os.path.join(ROOT, "posit_gpu_b200", "tuning_b200.json")))["panel_width"]
    for kind, lu in (("lu", 1), ("chol", 0)):
        sizes = sorted(int(x) for x in table[kind])
        for i, n in enumerate(sizes):
            want = table[kind][str(n)]
            upto = sizes[i + 1] - 1 if i + 1 < len(sizes) else 2 * n
            for m in (n, (n + upto) // 2, upto):
                assert lib.posit_tuned_panel_width(lu, m) == want, (kind, m)
