"""numpy restatement of the int8-slice arithmetic of safire_b200/csrc/islice*.cu (test infrastructure).

Every step of the device arithmetic is exact or a single round-to-nearest in FP64/FP32, so this
emulation reproduces the device results bit for bit:

  row exponent e: floor(log2 max|x|) - 6, plus one when 2^-e max|x| > 126
  slices of y = 2^-e x: q1 = rint(y), r = 256 (y - q1), q2 = rint(r), q3 = rint(256 (r - q2)),
  a q3 of +128 carried into q2, a q2 of +128 or more into q1
  product: groups g0 = q1 t1, g1 = q1 t2 + q2 t1, g2 = q1 t3 + q2 t2 + q3 t1 (exact integers),
  s = g0 + 2^-8 g1 + 2^-16 g2 (exact in FP64), out = fp32(s * 2^(eA + eB) * alpha)
"""
import numpy as np

PAIRS = {2: [(0, 0, 0), (0, 1, 1), (1, 0, 1)],
         3: [(0, 0, 0), (0, 1, 1), (1, 0, 1), (0, 2, 2), (1, 1, 2), (2, 0, 2)]}


def row_exponent(m):
    m = np.asarray(m, np.float64)
    _, ex = np.frexp(m)
    e = ex.astype(np.int64) - 7
    e = np.where(np.ldexp(m, -e) > 126.0, e + 1, e)
    return np.where(m > 0, e, 0).astype(np.int64)


def slices_at(X, e, ns):
    """the ns int8 slices (ns, R, K) of the rows of X (float64) at exponents e (R,)"""
    Y = np.ldexp(np.asarray(X, np.float64), -np.asarray(e)[:, None])
    a = np.rint(Y)
    r = (Y - a) * 256.0
    b = np.rint(r)
    q1, q2 = a.astype(np.int64), b.astype(np.int64)
    q3 = np.zeros_like(q1)
    if ns > 2:
        q3 = np.rint((r - b) * 256.0).astype(np.int64)
        c = q3 == 128
        q3[c] = -128
        q2[c] += 1
    c = q2 >= 128
    q2[c] -= 256
    q1[c] += 1
    out = np.stack([q1, q2, q3][:ns])
    assert out.min() >= -128 and out.max() <= 127
    return out


def slice_rows(X, ns):
    X = np.asarray(X, np.float64)
    e = row_exponent(np.max(np.abs(X), axis=1) if X.shape[1] else np.zeros(X.shape[0]))
    return slices_at(X, e, ns), e


def combine(groups, ea, eb, alpha=1.0):
    """fp32(s * 2^(ea + eb) * alpha) with s = g0 + 2^-8 g1 + 2^-16 g2, groups (ns, M, N) integer-valued"""
    s = groups[0].astype(np.float64)
    if len(groups) > 1:
        s = s + groups[1].astype(np.float64) * 2.0 ** -8
    if len(groups) > 2:
        s = s + groups[2].astype(np.float64) * 2.0 ** -16
    scale = np.ldexp(1.0, (ea[:, None] + eb[None, :]))
    return ((s * scale) * alpha).astype(np.float32)


def groups_of(qa, qb, ns):
    """exact group sums (ns, M, N) of the slice products qa (ns, M, K) x qb (ns, N, K)^T"""
    g = np.zeros((ns, qa.shape[1], qb.shape[1]))
    for i, j, grp in PAIRS[ns]:
        g[grp] += qa[i].astype(np.float64) @ qb[j].astype(np.float64).T  # integers < 2^53: exact
    return g


def gemm(A, B, ns, alpha=1.0, k0=0, k1=None):
    """C = A B^T over K in [k0, k1) as the device computes it (slices of the whole rows)"""
    qa, ea = slice_rows(A, ns)
    qb, eb = slice_rows(B, ns)
    k1 = A.shape[1] if k1 is None else k1
    return combine(groups_of(qa[:, :, k0:k1], qb[:, :, k0:k1], ns), ea, eb, alpha)


def cplx_b(A, V, ns):
    """C[c][w][a][j] = part c of sum_i A[w][a][i] V[w][j][i], with A and V taken through FP32"""
    W, N, M = A.shape
    Ar = A.real.astype(np.float32).astype(np.float64)
    Ai = A.imag.astype(np.float32).astype(np.float64)
    Vr = V.real.astype(np.float32).astype(np.float64)
    Vi = V.imag.astype(np.float32).astype(np.float64)
    out = np.zeros((2, W, N, M), np.float32)
    for w in range(W):
        ea = row_exponent(np.maximum(np.max(np.abs(Ar[w]), axis=1), np.max(np.abs(Ai[w]), axis=1)))
        ev = row_exponent(np.maximum(np.max(np.abs(Vr[w]), axis=1), np.max(np.abs(Vi[w]), axis=1)))
        qre, qim = slices_at(Ar[w], ea, ns), slices_at(Ai[w], ea, ns)
        qvr, qvi, qnvi = slices_at(Vr[w], ev, ns), slices_at(Vi[w], ev, ns), slices_at(-Vi[w], ev, ns)
        gre = groups_of(qre, qvr, ns) + groups_of(qim, qnvi, ns)
        gim = groups_of(qre, qvi, ns) + groups_of(qim, qvr, ns)
        out[0, w] = combine(gre, ea, ev)
        out[1, w] = combine(gim, ea, ev)
    return out
