"""CPU restatement of the 8-bit-digit split product (test infrastructure).

The device path (``csrc/gemm_split.cu``, TNT_PREC_INT8X) emulates each FP64
coupled-sector GEMM C = A B with exact integer tensor-core products.  This
module restates every step with numpy so the device output can be checked
bit for bit, not only within an error bound:

* every row of A and every column of B gets the power-of-two scale
  sigma = 2^e with amax = f 2^e, f in [0.5, 1) (``frexp``; 1 for a zero row);
* x' = x / sigma is rounded once to X = rint(x' 2^{8S-2}) (half to even) and
  cut into S balanced base-256 digits: d_0 in [-64, 64], d_s in [-128, 127];
* the digit products of each diagonal d = s + t < S are summed exactly over
  K chunks of 16384;
* per chunk, the diagonal sums are combined exactly in integers, in two
  parts: hi = sum_{d<H} acc_d 256^{H-1-d} and lo = sum_{H<=d<S} acc_d
  256^{S-1-d} with H = min(S, 3); the FP64 value v = hi + lo 2^{-8(S-H)} is
  rounded once, and v times (sigma_row 2^{-12-8(H-1)} alpha) tau_col is
  written (chunk 0) or added (later chunks) into C.  With beta != 0 the device
  fuses beta C + value into one FMA, which numpy rounds twice, so bit-exact
  checks use beta = 0.

The split scheme is this project's own (the reference multiplies in plain
FP64); the reference's part of the product is the per-sector job table of
``Rank2GemmBatchJob`` (tenet-operations/src/fusion_replay.rs:518-528), which
``replay_compose_i8`` walks the same way ``tests.helpers.replay_compose`` does.
"""

from __future__ import annotations

import numpy as np

KCHUNK = 16384


def pow2_scale(amax: np.ndarray) -> np.ndarray:
    amax = np.asarray(amax, dtype=np.float64)
    pos = amax > 0
    e = np.frexp(np.where(pos, amax, 1.0))[1]
    return np.where(pos, np.ldexp(1.0, e), 1.0)


def digits8(xp: np.ndarray, S: int):
    """X = rint(x' 2^{8S-2}) and its S balanced base-256 digits (d_0 first)."""
    X = np.rint(np.ldexp(np.asarray(xp, dtype=np.float64), 8 * S - 2)).astype(np.int64)
    C = 0
    for _ in range(S - 1):
        C = C * 256 + 128
    Y = X + C
    out = []
    for s in range(S):
        u = Y >> (8 * (S - 1 - s))  # arithmetic shift: floor division
        out.append(u if s == 0 else (u & 255) - 128)
    return X, out


def digits8_from_bits(xp: np.ndarray, S: int):
    """The device's route to the same digits: v = x' 2^{8S-2} + (1.5 2^52 + C)
    rounded once; byte b of v's bit pattern is byte b of Y = X + C, so digit
    S-1-b is that byte (minus 128 for the low digits, as a signed byte for the
    top one)."""
    C = 0
    for _ in range(S - 1):
        C = C * 256 + 128
    magic = 6755399441055744.0 + float(C)
    v = np.ldexp(np.asarray(xp, dtype=np.float64), 8 * S - 2) + magic  # exact product, one rounding
    bits = v.view(np.uint64)
    out = []
    for s in range(S):
        b = S - 1 - s
        byte = ((bits >> np.uint64(8 * b)) & np.uint64(255)).astype(np.int64)
        out.append(np.where(byte >= 128, byte - 256, byte) if s == 0 else byte - 128)
    return out


def split_product_i8(A: np.ndarray, B: np.ndarray, S: int, alpha: float = 1.0,
                     beta: float = 0.0, C0: np.ndarray | None = None) -> np.ndarray:
    """Device value of alpha A B + beta C0 (A: m x k, B: k x n); bit-exact for beta = 0."""
    m, k = A.shape
    n = B.shape[1]
    if k == 0:
        return np.zeros((m, n)) if beta == 0.0 else beta * C0
    sa = pow2_scale(np.abs(A).max(axis=1))
    sb = pow2_scale(np.abs(B).max(axis=0))
    _, da = digits8(A / sa[:, None], S)
    _, db = digits8(B / sb[None, :], S)
    H = min(S, 3)
    sr = (sa * 2.0 ** (-12 - 8 * (H - 1))) * alpha
    out = None
    for c0 in range(0, k, KCHUNK):
        c1 = min(k, c0 + KCHUNK)
        acc = []
        for d in range(S):
            acc.append(sum(da[s][:, c0:c1] @ db[d - s][c0:c1, :] for s in range(d + 1)))  # exact int64
        hi = np.zeros_like(acc[0])
        for d in range(H):
            hi = hi * 256 + acc[d]
        lo = np.zeros_like(acc[0])
        for d in range(H, S):
            lo = lo * 256 + acc[d]
        v = hi.astype(np.float64) + lo.astype(np.float64) * 2.0 ** (-8 * (S - H))  # exact parts, one rounding
        val = (sr[:, None] * sb[None, :]) * v
        if out is None:
            out = val if beta == 0.0 else beta * C0 + val
        else:
            out = out + val
    return out


def replay_compose_i8(jobs, a, b, c_size, S, alpha=1.0, beta=0.0, c0=None):
    """The device's int8-digit compose over a plan's job table."""
    c = np.zeros(c_size) if c0 is None else np.array(c0, dtype=np.float64)
    for m, n, k, ao, bo, co, lda, ldb, ldc in jobs:
        if m == 0 or n == 0:
            continue
        view = c[co: co + ldc * n].reshape(n, ldc).T[:m]
        if k == 0:
            view[:] = 0.0 if beta == 0.0 else beta * view
            continue
        Am = a[ao: ao + lda * k].reshape(k, lda).T[:m]
        Bm = b[bo: bo + ldb * n].reshape(n, ldb).T[:k]
        view[:] = split_product_i8(Am, Bm, S, alpha, beta, view.copy())
    return c
