"""The integer forward contraction's host-side arithmetic, restated on the
CPU (mz_fm.cuh / mz_fm8.cuh): balanced base-256 digits of 31-bit integers,
the 128-byte-swizzled K-major block layout of the moments' and the
candidates' digits, the ten digit-pair MMAs summed per weight class (what
tcgen05.mma.kind::i8 adds exactly in 32 bits), the FP64 epilogue, and the
adjoint's dequantised operand read back from 16-slot sub-tiles.  The device
result against FP64 is tests/test_gpu_moments.py's."""
import math

import numpy as np

TM, D8, NC, DIG = 128, 256, 64, 4
XBLK, KBLK = TM * 128, NC * 128
STAGE = DIG * XBLK
SHIFT = 30
PAIRS = [(0, 0), (0, 1), (1, 0), (0, 2), (1, 1), (2, 0), (0, 3), (1, 2), (2, 1), (3, 0)]


def sw128(r, k):
    return (r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 4) ^ r) & 7) << 4) + (k & 15)


def x8_block(T, t, kb, l):
    return (((T * 3 + t) * 2 + kb) * DIG + l) * XBLK


def k8_block(gy, s, nt, kb, l):
    return (((gy * nt + s) * 2 + kb) * DIG + l) * KBLK


def digits(v):
    d = [0] * DIG
    for l in range(DIG - 1, 0, -1):
        lo = ((v + 128) & 255) - 128
        d[l] = lo
        v = (v - lo) // 256
    d[0] = v
    return d


def exponent(m):
    if not m > 0:
        return 0
    return max(-100, min(100, math.frexp(m)[1]))


def test_digits_round_trip_and_ranges():
    rng = np.random.default_rng(0)
    for v in list(rng.integers(-2 ** 30, 2 ** 30, 2000)) + [2 ** 30, -2 ** 30, 0, 1, -1, 127, -128, 255]:
        d = digits(int(v))
        assert -64 <= d[0] <= 64 and all(-128 <= x <= 127 for x in d[1:])
        assert sum(d[l] * 256 ** (DIG - 1 - l) for l in range(DIG)) == v


def test_swizzle_is_a_permutation_of_each_block():
    offs = {sw128(r, k) for r in range(TM) for k in range(128)}
    assert offs == set(range(XBLK))
    # 4-byte groups of a feature quad stay contiguous (the adjoint reads them as words)
    for r in range(16):
        for d in range(0, 128, 4):
            assert [sw128(r, d + b) for b in range(4)] == [sw128(r, d) + b for b in range(4)]


def _build(rng, nt, D, Q, CG):
    X = rng.normal(size=(3, Q, D)) * np.exp(rng.normal(size=(3, Q, 1)) * 3)
    X[:, Q - 20:, :] = 0.0
    K = rng.normal(size=(nt, CG, D)) * np.exp(rng.normal(size=(nt, CG, 1)))
    ntile8 = Q // TM
    X8 = np.zeros(ntile8 * 3 * 2 * STAGE, np.int8)
    xe = np.zeros(4 * Q, np.int8)
    for t in range(3):
        for q in range(Q):
            e = exponent(np.max(np.abs(X[t, q])))
            xe[q * 4 + t] = e
            T, r = divmod(q, TM)
            for d in range(D):
                dg = digits(int(np.rint(math.ldexp(X[t, q, d], SHIFT - e))))
                for l in range(DIG):
                    X8[x8_block(T, t, d >> 7, l) + sw128(r, d & 127)] = dg[l]
    K8 = np.zeros(nt * 2 * DIG * KBLK, np.int8)
    ke = np.zeros((nt, NC), int)
    for s in range(nt):
        for c in range(NC):
            e = exponent(np.max(np.abs(K[s, c]))) if c < CG else 0
            ke[s, c] = e
            for d in range(D8):
                kv = K[s, c, d] if (c < CG and d < D) else 0.0
                dg = digits(int(np.rint(math.ldexp(kv, SHIFT - e))))
                for l in range(DIG):
                    K8[k8_block(0, s, nt, d >> 7, l) + sw128(c, d & 127)] = dg[l]
    return X, K, X8, xe, K8, ke


def test_class_sums_and_epilogue_match_fp64():
    rng = np.random.default_rng(1)
    nt, D, Q, CG = 2, 240, 256, 64
    X, K, X8, xe, K8, ke = _build(rng, nt, D, Q, CG)
    idxA = np.array([[sw128(r, k) for k in range(128)] for r in range(TM)])
    idxB = np.array([[sw128(c, k) for k in range(128)] for c in range(NC)])
    worst = 0.0
    for T, s in ((0, 0), (1, 1)):
        for t in range(3):
            acc = np.zeros((4, TM, NC), np.int64)
            for kb in range(2):
                for i, j in PAIRS:
                    A = X8[x8_block(T, t, kb, i) + idxA].astype(np.int64)
                    B = K8[k8_block(0, s, nt, kb, j) + idxB].astype(np.int64)
                    acc[i + j] += A @ B.T
            assert np.max(np.abs(acc)) < 2 ** 31
            for r in range(TM):
                q = T * TM + r
                a = (acc[0, r] * 2.0 ** 48 + acc[1, r] * 2.0 ** 40) + (acc[2, r] * 2.0 ** 32 + acc[3, r] * 2.0 ** 24)
                y = a * 2.0 ** (int(xe[q * 4 + t]) - SHIFT) * 2.0 ** (ke[s].astype(float) - SHIFT)
                scale = np.max(np.abs(X[t, q])) * np.max(np.abs(K[s]), axis=1) + 1e-300
                worst = max(worst, float(np.max(np.abs(y[:CG] - X[t, q] @ K[s].T) / scale)))
    assert worst <= 2e-7, worst


def test_adjoint_sub_tile_dequantisation():
    rng = np.random.default_rng(2)
    nt, D, Q, CG, SUB, Dpad = 1, 240, 128, 8, 16, 240
    X, K, X8, xe, K8, ke = _build(rng, nt, D, Q, CG)
    worst = 0.0
    for qb in range(0, Q, SUB):
        T, r0 = divmod(qb, TM)
        raw = np.zeros(3 * 2 * DIG * 2048, np.int8)
        for blk in range(3 * 2 * DIG):
            src = T * 3 * 2 * STAGE + blk * XBLK + (r0 >> 3) * 1024
            raw[blk * 2048:(blk + 1) * 2048] = X8[src:src + 2048]
        for t in range(3):
            for j in range(SUB):
                sc = 2.0 ** (int(xe[(qb + j) * 4 + t]) - SHIFT)
                m = np.max(np.abs(X[t, qb + j]))
                for d in range(0, Dpad, 4):
                    o = sw128(j, d & 127)
                    for b in range(4):
                        v = 0
                        for l in range(DIG):
                            v = v * 256 + int(raw[((t * 2 + (d >> 7)) * DIG + l) * 2048 + o + b])
                        x = float(np.float32(v * sc))
                        ref = X[t, qb + j, d + b] if d + b < D else 0.0
                        if m > 0:
                            worst = max(worst, abs(x - ref) / m)
    assert worst <= 1.2e-7, worst


ZBLK = NC * 128
SPAN = 8  # tiles per exponent span of the adjoint's operand


def digits_np(v):
    """digits() over an int64 array: [DIG, ...] most significant first."""
    d = np.zeros((DIG,) + v.shape, np.int64)
    for l in range(DIG - 1, 0, -1):
        lo = ((v + 128) & 255) - 128
        d[l] = lo
        v = (v - lo) >> 8
    d[0] = v
    return d


def test_adjoint_class_sums_read_moments_mn_major():
    """The adjoint's MMAs read the moments' digit blocks as an MN-major
    operand (features along M, slots along K) and Z = 2^(e_q - 30) Ybar as
    K-major digit blocks written by the converter warps, with one exponent
    per (span of SPAN tiles, candidate) from the pre pass's bound on the FP32
    exponent fields; the class sums run over a whole span exactly in 32 bits,
    and the read-out at the span's end gives Kbar = sum_{t,q} X Ybar."""
    rng = np.random.default_rng(3)
    nt, D, CG = 1, 240, 64
    ntile8 = SPAN + 2  # two spans, the second one partial
    Q = ntile8 * TM
    X, K, X8, xe, K8, ke = _build(rng, nt, D, Q, CG)
    Yb = (rng.normal(size=(Q, 3, CG)) * np.exp(rng.normal(size=(Q, 1, 1)) * 2)).astype(np.float32)
    eq = xe.reshape(Q, 4)[:, :3].astype(np.int64)
    # the pre pass's bound: |Ybar| < 2^(field - 126), so |Z| < 2^(field - 126 + e_q - 30)
    field = ((Yb.view(np.uint32) >> 23) & 255).astype(np.int64)
    zexp = np.where(Yb != 0, field - 126 + eq[:, :, None] - SHIFT, -(2 ** 31))
    nspan = (ntile8 + SPAN - 1) // SPAN
    zm = np.full((nspan, NC), -(2 ** 31), np.int64)
    for sp in range(nspan):
        zm[sp, :CG] = zexp[sp * SPAN * TM:(sp + 1) * SPAN * TM].max(axis=(0, 1))
    e = np.where(zm > -1000, np.maximum(-100, zm), 0)
    # the converters: Z_int = rint(Ybar 2^(e_q - e)), one rounding, |Z_int| <= 2^30
    sp_of_q = np.arange(Q) // (SPAN * TM)
    Zi = np.rint(Yb.astype(np.float64) * np.exp2((eq[:, :, None] - e[sp_of_q][:, None, :CG]).astype(np.float64)))
    Zi = Zi.astype(np.int64)
    assert np.max(np.abs(Zi)) <= 2 ** 30
    Zd = digits_np(Zi)  # [DIG][Q][3][CG]
    assert np.all(np.abs(Zd[0]) <= 64) and np.all((Zd[1:] >= -128) & (Zd[1:] <= 127))
    # A[d][q]: the moments' block read MN-major, element (d, q) at sw128(q, d);
    # B[c][q]: the converters' 16-byte chunk of row c holds slots 16 g .. 16 g + 15
    idxA = np.array([[sw128(q, d) for q in range(TM)] for d in range(128)])
    idxB = np.array([[sw128(c, q) for q in range(TM)] for c in range(NC)])
    assert all(sw128(c, 16 * g) + k == sw128(c, 16 * g + k) for c in range(NC) for g in range(8) for k in range(16))
    Kbar = np.zeros((256, NC))
    acc = np.zeros((2, 4, 128, NC), np.int64)
    for T in range(ntile8):
        for t in range(3):
            stage = np.zeros((DIG, ZBLK), np.int8)
            for l in range(DIG):
                img = np.zeros((NC, TM), np.int64)
                img[:CG] = Zd[l, T * TM:(T + 1) * TM, t, :].T
                stage[l][idxB] = img
            for kb in range(2):
                for i, j in PAIRS:
                    A = X8[x8_block(T, t, kb, i) + idxA].astype(np.int64)
                    B = stage[j][idxB].astype(np.int64)
                    acc[kb, i + j] += A @ B.T
        if (T + 1) % SPAN == 0 or T + 1 == ntile8:  # the segment's read-out
            assert np.max(np.abs(acc)) < 2 ** 31
            sc = np.exp2((e[T // SPAN] - SHIFT).astype(np.float64))
            for kb in range(2):
                a = (acc[kb, 0] * 2.0 ** 48 + acc[kb, 1] * 2.0 ** 40) + (acc[kb, 2] * 2.0 ** 32 + acc[kb, 3] * 2.0 ** 24)
                Kbar[kb * 128:(kb + 1) * 128] += a * sc
            acc[:] = 0
    ref = np.einsum("tqd,qtc->dc", X, Yb.astype(np.float64))
    # the two quantisations bound the error: |Z - Z'| <= 2^(e_span - 31) per
    # element against the unscaled moment digits, |X - X'| <= 2^(e_q - 31)
    # against Ybar (the dropped digit classes weigh 2^-38 of these)
    Xint = np.zeros((3, Q, D))
    for T in range(ntile8):
        for t in range(3):
            for kb in range(2):
                v = sum(X8[x8_block(T, t, kb, l) + idxA].astype(np.float64) * 256.0 ** (DIG - 1 - l) for l in range(DIG))
                d1 = min(D, (kb + 1) * 128)
                if d1 > kb * 128:
                    Xint[t, T * TM:(T + 1) * TM, kb * 128:d1] = v.T[:, :d1 - kb * 128]
    zq = np.exp2((e[sp_of_q][:, :CG] - SHIFT - 1).astype(np.float64))  # [Q][CG]
    xq = np.exp2((eq - SHIFT - 1).astype(np.float64))  # [Q][3]
    bound = np.einsum("tqd,qc->dc", np.abs(Xint), zq) + np.einsum("tqd,qt,qtc->dc", np.ones_like(X), xq,
                                                                       np.abs(Yb.astype(np.float64)))
    scale = np.einsum("tqd,qtc->dc", np.abs(X), np.abs(Yb.astype(np.float64)))
    err = np.abs(Kbar[:D, :CG] - ref)
    assert np.all(err <= 1.01 * bound + 1e-12 * scale), np.max(err / bound)
    # against the magnitudes: spans of widely varying rows (this data spans a
    # factor 1e4 within a span) lose bits on their small rows, never on the largest
    assert np.max(err / scale) <= 2e-5


def _byte_perm(x, y, sel):
    b = [(x >> (8 * i)) & 255 for i in range(4)] + [(y >> (8 * i)) & 255 for i in range(4)]
    return sum(b[(sel >> (4 * i)) & 7] << (8 * i) for i in range(4))


def test_converter_digit_bytes_and_transpose():
    """The adjoint's converters take the balanced base-256 digits of
    |Z_int| <= 2^30 as the bytes of (Z_int + 0x808080) ^ 0x808080 and gather
    one digit of four slots per word with a 4 x 4 byte transpose
    (__byte_perm selectors 0x5140 / 0x7362, then 0x5410 / 0x7632)."""
    rng = np.random.default_rng(5)
    edge = [2 ** 30, -(2 ** 30), 0, 1, -1, 127, -128, 128, -129, 255, -256, 32767, -32769]
    vals = [int(v) for v in rng.integers(-(2 ** 30), 2 ** 30 + 1, 4000)] + edge * 4
    for i in range(0, len(vals) - 3, 4):
        z = vals[i:i + 4]
        v = [((x + 0x808080) ^ 0x808080) & 0xFFFFFFFF for x in z]
        ablo, abhi = _byte_perm(v[0], v[1], 0x5140), _byte_perm(v[0], v[1], 0x7362)
        cdlo, cdhi = _byte_perm(v[2], v[3], 0x5140), _byte_perm(v[2], v[3], 0x7362)
        w = {3: _byte_perm(ablo, cdlo, 0x5410), 2: _byte_perm(ablo, cdlo, 0x7632),
             1: _byte_perm(abhi, cdhi, 0x5410), 0: _byte_perm(abhi, cdhi, 0x7632)}
        for u, x in enumerate(z):
            d = digits(x)
            for l in range(DIG):
                assert (w[l] >> (8 * u)) & 255 == d[l] & 255, (x, l)
