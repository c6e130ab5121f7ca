"""FP64 accuracy reports for posit32 solves, computed on the GPU.

The reference's drivers measure accuracy against FP64 LAPACK on the same inputs
(main_lu_check.cpp:152-247, main_cholesky_check.cpp): relative residual ||b - A x|| / ||b||
and the error against the known solution.  Here the posit32-valued A and b are converted
exactly to FP64 (posit_to_double_dev), solved in FP64 on the GPU (torch.linalg, i.e.
cuSOLVER: the only floating-point work on the device), and the posit32 solution x is
compared with it and with the known x_true:

    forward_error   ||x - x_true||_2 / ||x_true||_2
    backward_error  ||b - A x||_2 / (||A||_F ||x||_2)       (A, b, x exact in FP64)
    residual        ||b - A x||_2 / ||b||_2                  (the drivers' figure)
    fp64_forward_error of the FP64 solution, for scale.
"""
import torch

from . import to_double_dev


def _f64(t):
    return to_double_dev(t.contiguous().view(torch.int32))


def solve_report(A, b, x, x_true=None, n=None, spd=False):
    """A: n x n posit32 (4-byte CUDA tensor, column-major flat), b, x (and x_true): n
    posit32 vectors on the same device.  Returns a dict of FP64 error figures."""
    n = n or b.numel()
    A64 = _f64(A).reshape(n, n).t()  # column-major -> row-major view
    b64, x64 = _f64(b), _f64(x)
    r = b64 - A64 @ x64
    out = {
        "residual": float(r.norm() / b64.norm()),
        "backward_error": float(r.norm() / (A64.norm() * x64.norm())),
    }
    if spd:
        L = torch.linalg.cholesky(A64)
        ref = torch.cholesky_solve(b64.unsqueeze(1), L).squeeze(1)
    else:
        ref = torch.linalg.solve(A64, b64)
    out["fp64_vs_posit"] = float((x64 - ref).norm() / ref.norm())
    if x_true is not None:
        xt = _f64(x_true)
        out["forward_error"] = float((x64 - xt).norm() / xt.norm())
        out["fp64_forward_error"] = float((ref - xt).norm() / xt.norm())
    return out
