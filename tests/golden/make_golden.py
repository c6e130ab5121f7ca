"""Generate the golden vectors in this folder from the REFERENCE'S OWN CODE.

The reference has no tests or fixtures of its own, so the golden vectors are outputs
of its sources compiled here (``oracle/_ref/libposit_ref.so``, built by
``oracle/build_oracle.py`` from ``libRpack/kernel_entry.cl`` and the untouched libRpack
CPU routines).  Run from the repository root where the reference tree is present:

    python oracle/build_oracle.py && python tests/golden/make_golden.py

Outputs:
  ops.npz     p32_add / p32_mul (kernel_entry.cl:370-538) on special values, random
              patterns, near-cancelling pairs and long-regime operands
  rgemm.npz   Rgemm (Rgemm.cpp:62-251) on small shapes, all four transpose cases,
              padded leading dimensions, special alpha/beta, zeros/NaR/extremes
  lapack.npz  Rgetrf / Rgetrs / Rpotrf / Rpotrs (nb override) on small systems
  hashes.json SHA-256 of Rgemm outputs on larger seeded problems (config-1 512^3 NN and
              a 256^3 case per transpose), with the recipe that regenerates the inputs
  factor_hashes.json
              SHA-256 of the reference's Rgetrf/Rgetrs and Rpotrf/Rpotrs results on the
              seeded n = 1024 and 4096 systems (nb = 256); `... make_golden.py factors`
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402
from tests import posit_data as pd  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
ONE, NAR, M1 = oracle.P32_ONE, oracle.P32_NAR, oracle.P32_MINUS_ONE


def ref_lib():
    if oracle.ref is None:
        raise SystemExit("oracle/_ref/libposit_ref.so not built: run oracle/build_oracle.py "
                         "where the reference tree is present")
    return oracle.ref


def make_ops(ref):
    rng = np.random.default_rng(20250101)
    specials = np.array([0, NAR, 1, 2, 3, 0x7FFFFFFF, 0x7FFFFFFE, 0x7FFFFFFD, ONE, M1,
                         0x80000001, 0xFFFFFFFF, 0xFFFFFFFE, 0x48000000, 0x38000000,
                         0x3FFFFFFF, 0x40000001, 0x00800000, 0x7F800000], dtype=np.uint32)
    a = [np.repeat(specials, specials.size)]
    b = [np.tile(specials, specials.size)]
    n = 3000
    a.append(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32))
    b.append(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32))
    x = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    d = rng.integers(-64, 64, n).astype(np.int64)
    a.append(x)
    b.append(((0 - x.astype(np.int64) + d) & 0xFFFFFFFF).astype(np.uint32))
    ext = rng.integers(0, 2**10, n).astype(np.uint32)
    ext = np.where(rng.integers(0, 2, n) == 1, (0x7FFFFFFF - ext).astype(np.uint32), ext)
    ext = np.where(rng.integers(0, 2, n) == 1, (0 - ext.astype(np.int64)) & 0xFFFFFFFF, ext).astype(np.uint32)
    a.append(ext)
    b.append(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32))
    a.append(pd.uniform(rng, (n,)))
    b.append(pd.uniform(rng, (n,)))
    a = np.concatenate(a)
    b = np.concatenate(b)
    add = np.empty_like(a)
    mul = np.empty_like(a)
    ref.ref_p32_add_n(a, b, add, a.size)
    ref.ref_p32_mul_n(a, b, mul, a.size)
    np.savez_compressed(os.path.join(OUT, "ops.npz"), a=a, b=b, add=add, mul=mul)
    return a.size


def gemm_cases():
    rng = np.random.default_rng(777)
    cases = []
    shapes = [(1, 1, 1), (3, 2, 5), (7, 5, 9), (16, 16, 16), (33, 17, 65), (40, 31, 7)]
    scal = [(ONE, 0), (ONE, ONE), (M1, ONE), (oracle.p32(0.75), oracle.p32(-1.5)),
            (0, oracle.p32(0.5)), (0, 0)]
    idx = 0
    for ta, tb in (("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")):
        for (m, n, k) in shapes:
            for (alpha, beta) in scal[(idx % 3):(idx % 3) + 4]:
                kind = "wide" if idx % 5 == 4 else "uniform"
                ar, ac = (m, k) if ta == "N" else (k, m)
                br, bc = (k, n) if tb == "N" else (n, k)
                pad = idx % 3
                lda, ldb, ldc = ar + pad, br + pad, m + pad
                A = pd.colmajor(rng, ar, ac, lda, kind)
                B = pd.colmajor(rng, br, bc, ldb, kind)
                C = pd.colmajor(rng, m, n, ldc, kind)
                if idx % 7 == 3:
                    for buf in (A, B, C):
                        j = rng.integers(0, buf.size, size=max(1, buf.size // 10))
                        buf[j[0::3]] = 0
                        buf[j[1::3]] = 0x7FFFFFFF
                        buf[j[2::3]] = 1
                if idx % 11 == 5:
                    A[rng.integers(0, A.size)] = NAR
                cases.append(dict(ta=ta, tb=tb, m=m, n=n, k=k, alpha=alpha, beta=beta,
                                  A=A, lda=lda, B=B, ldb=ldb, C=C, ldc=ldc))
                idx += 1
    return cases


def make_rgemm(ref):
    cases = gemm_cases()
    arrays = {}
    meta = []
    for i, c in enumerate(cases):
        out = c["C"].copy()
        ref.ref_rgemm(c["ta"].encode(), c["tb"].encode(), c["m"], c["n"], c["k"], c["alpha"],
                      c["A"], c["lda"], c["B"], c["ldb"], c["beta"], out, c["ldc"])
        arrays[f"A{i}"] = c["A"]
        arrays[f"B{i}"] = c["B"]
        arrays[f"C{i}"] = c["C"]
        arrays[f"out{i}"] = out
        meta.append([ord(c["ta"]), ord(c["tb"]), c["m"], c["n"], c["k"], c["alpha"], c["beta"],
                     c["lda"], c["ldb"], c["ldc"]])
    arrays["meta"] = np.array(meta, dtype=np.int64)
    np.savez_compressed(os.path.join(OUT, "rgemm.npz"), **arrays)
    return len(cases)


def spd(rng, n):
    M = rng.uniform(-1, 1, size=(n, n))
    return oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))


def make_lapack(ref):
    rng = np.random.default_rng(4242)
    arrays = {}
    meta = []
    for i, (n, nb, nrhs) in enumerate([(1, 2, 1), (5, 2, 2), (16, 4, 1), (37, 8, 3), (64, 16, 2), (70, 32, 1)]):
        A = oracle.from_double(rng.uniform(-1, 1, size=n * n))
        b = oracle.from_double(rng.uniform(-1, 1, size=n * nrhs))
        lu = A.copy()
        ipiv = np.zeros(n, dtype=np.int32)
        info = ref.ref_rgetrf(n, n, lu, n, ipiv, nb)
        x = b.copy()
        ref.ref_rgetrs(b"N", n, nrhs, lu, n, ipiv, x, n)
        S = spd(rng, n)
        ch = S.copy()
        cinfo = ref.ref_rpotrf(b"L", n, ch, n, nb)
        xs = b.copy()
        ref.ref_rpotrs(b"L", n, nrhs, ch, n, xs, n)
        chu = S.copy()
        uinfo = ref.ref_rpotrf(b"U", n, chu, n, nb)
        arrays.update({f"A{i}": A, f"b{i}": b, f"lu{i}": lu, f"ipiv{i}": ipiv, f"x{i}": x,
                       f"S{i}": S, f"chl{i}": ch, f"xs{i}": xs, f"chu{i}": chu})
        meta.append([n, nb, nrhs, info, cinfo, uinfo])
    arrays["meta"] = np.array(meta, dtype=np.int64)
    np.savez_compressed(os.path.join(OUT, "lapack.npz"), **arrays)
    return len(meta)


def hash_cases():
    """Larger problems whose inputs are regenerated from a seed (see regen_inputs)."""
    out = [dict(name="config1_nn_512", ta="N", tb="N", n=512, seed=20240101, alpha=oracle.p32(1.0),
                beta=oracle.p32(0.5))]
    for ta, tb in (("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")):
        out.append(dict(name=f"{ta}{tb}_256_m1_1", ta=ta, tb=tb, n=256, seed=31337, alpha=M1, beta=ONE))
    return out


def regen_inputs(case):
    """Square n x n A, B, C, uniform [-1,1] from default_rng(seed), drawn A then B then C."""
    rng = np.random.default_rng(case["seed"])
    n = case["n"]
    return pd.uniform(rng, (n * n,)), pd.uniform(rng, (n * n,)), pd.uniform(rng, (n * n,))


def make_hashes(ref):
    res = []
    for c in hash_cases():
        A, B, C = regen_inputs(c)
        n = c["n"]
        ref.ref_rgemm(c["ta"].encode(), c["tb"].encode(), n, n, n, c["alpha"], A, n, B, n, c["beta"], C, n)
        res.append(dict(c, sha256=hashlib.sha256(C.tobytes()).hexdigest(),
                        input_sha256=hashlib.sha256(regen_inputs(c)[0].tobytes()).hexdigest()))
    with open(os.path.join(OUT, "hashes.json"), "w") as f:
        json.dump(res, f, indent=1)
    return len(res)


def factor_cases():
    """Config-3 factorizations: GE U[-1,1] for LU, SPD M*M^T/n + I for Cholesky, nb = 256,
    b = A*x_true with x_true U[-1,1]."""
    return [dict(name=f"lu_{n}", kind="lu", n=n, nb=256, seed=3000 + n) for n in (1024, 4096)] + \
           [dict(name=f"chol_{n}", kind="chol", n=n, nb=256, seed=5000 + n) for n in (1024, 4096)]


def regen_factor_inputs(case):
    """A (column-major n x n) and x_true, from default_rng(seed): for LU A ~ U[-1,1]; for
    Cholesky M ~ U[-1,1] then A = M*M^T/n + I formed in FP64; then x_true ~ U[-1,1]."""
    rng = np.random.default_rng(case["seed"])
    n = case["n"]
    if case["kind"] == "lu":
        A = oracle.from_double(rng.uniform(-1.0, 1.0, n * n))
    else:
        M = rng.uniform(-1.0, 1.0, (n, n))
        A = oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))
    x = oracle.from_double(rng.uniform(-1.0, 1.0, n))
    return A, x


def make_factor_hashes(ref, names=None):
    """SHA-256 of the reference's CPU factors, pivots and solutions (can take minutes)."""
    out_path = os.path.join(OUT, "factor_hashes.json")
    res = json.load(open(out_path)) if os.path.exists(out_path) else {}
    for c in factor_cases():
        if names and c["name"] not in names:
            continue
        A, x = regen_factor_inputs(c)
        n = c["n"]
        b = np.zeros(n, np.uint32)
        ref.ref_rgemv(b"N", n, n, oracle.P32_ONE, A, n, x, 1, 0, b, 1)  # b = A*x (Rgemv.cpp:152-162)
        F = A.copy()
        rhs = b.copy()
        if c["kind"] == "lu":
            ipiv = np.zeros(n, np.int32)
            info = ref.ref_rgetrf(n, n, F, n, ipiv, c["nb"])
            ref.ref_rgetrs(b"N", n, 1, F, n, ipiv, rhs, n)
            extra = {"ipiv_sha256": hashlib.sha256(ipiv.tobytes()).hexdigest()}
        else:
            info = ref.ref_rpotrf(b"L", n, F, n, c["nb"])
            ref.ref_rpotrs(b"L", n, 1, F, n, rhs, n)
            extra = {}
        res[c["name"]] = dict(c, info=int(info), A_sha256=hashlib.sha256(A.tobytes()).hexdigest(),
                              b_sha256=hashlib.sha256(b.tobytes()).hexdigest(),
                              factor_sha256=hashlib.sha256(F.tobytes()).hexdigest(),
                              x_sha256=hashlib.sha256(rhs.tobytes()).hexdigest(), **extra)
        with open(out_path, "w") as f:
            json.dump(res, f, indent=1)
        print("factor hash", c["name"], flush=True)
    return len(res)


def main():
    import sys
    ref = ref_lib()
    if len(sys.argv) > 1 and sys.argv[1] == "factors":
        print("factors", make_factor_hashes(ref, sys.argv[2:] or None))
        return
    print("ops", make_ops(ref))
    print("rgemm", make_rgemm(ref))
    print("lapack", make_lapack(ref))
    print("hashes", make_hashes(ref))


if __name__ == "__main__":
    main()
