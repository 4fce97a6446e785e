"""The exactness arguments behind two rewrites of the device arithmetic,
checked on the CPU with the same operations in numpy:

* the key switch's CRT high digit (`high_digit`, dnspir_b200/csrc/chain.cu;
  partial_gal's decomposition, crates/pir/src/base_pir.rs:541-571) computed in
  double precision equals the 64-bit integer formula on random inputs and on
  every rounding boundary near 2^26-multiples and near q/2;
* the forward butterfly without input reduction (`ct`, ntt.cuh) keeps an
  11-stage transform below 26p < 2^31 from inputs below 4p (each stage adds
  at most 2p), and the Shoup product by one plus one subtraction
  (`canon`) then gives the exact residues.
The GPU parity tests check the kernels themselves against the oracle."""
import numpy as np

P1 = (1 << 26) - (1 << 12) + 1
P2 = (1 << 25) - (1 << 12) + 1
QQ = P1 * P2


def digit_int(x1, x2):
    v = x1.astype(np.int64) * P2 + x2.astype(np.int64) * P1  # < 2^52
    v = np.where(v >= QQ, v - QQ, v)
    x = np.where(v > QQ // 2, v - QQ, v)
    return (x + (1 << 25)) >> 26


def digit_double(x1, x2):
    v = x1.astype(np.float64) * float(P2) + x2.astype(np.float64) * float(P1)
    v = np.where(v >= float(QQ), v - float(QQ), v)
    v = np.where(v > float(QQ // 2), v - float(QQ), v)
    return np.floor(v * (1.0 / (1 << 26)) + 0.5).astype(np.int64)


def test_high_digit_double_equals_integer_formula():
    rng = np.random.default_rng(5)
    x1 = rng.integers(0, P1, 1_000_000)
    x2 = rng.integers(0, P2, 1_000_000)
    assert np.array_equal(digit_int(x1, x2), digit_double(x1, x2))
    # values whose centred lift sits on or next to a rounding boundary, and
    # next to the centring threshold q/2
    i2, i1 = pow(P2, -1, P1), pow(P1, -1, P2)
    targets = []
    for k in range(-3000, 3000):
        b = k * (1 << 26) - (1 << 25)
        targets += [b - 1, b, b + 1]
    targets += [QQ // 2 - 1, QQ // 2, QQ // 2 + 1, QQ - 1, 0]
    v = np.array([t % QQ for t in targets], dtype=object)
    x1 = np.array([(int(t) * i2) % P1 for t in v], dtype=np.int64)
    x2 = np.array([(int(t) * i1) % P2 for t in v], dtype=np.int64)
    assert np.array_equal(digit_int(x1, x2), digit_double(x1, x2))


def _lazy_mul(x, w, wq, p):
    # x * w - floor(x * wq / 2^32) * p, in 32-bit arithmetic as on the device
    return (x * w - ((x * wq) >> 32) * p) & 0xFFFFFFFF


def test_lazy_forward_butterflies_stay_below_2_31():
    # an 11-stage Cooley-Tukey network (length 2048) of the device's forward
    # butterfly (x, y) -> (x + t, x - t + 2p), t = Shoup product of y, on
    # inputs near 4p and random twiddles: no value reaches 26p, and the
    # canonicalised outputs equal the same network computed exactly mod p
    rng = np.random.default_rng(9)
    for p in (P1, P2):
        one_q = (1 << 32) // p
        x = rng.integers(4 * p - 64, 4 * p, 2048).astype(object)
        exact = [int(v) % p for v in x]
        x = [int(v) for v in x]
        top = 0
        for s in range(11):
            d = 1024 >> s
            for blk in range(1 << s):
                w = int(rng.integers(0, p))
                wq = (w << 32) // p
                for r in range(d):
                    i, j = blk * 2 * d + r, blk * 2 * d + r + d
                    t = _lazy_mul(x[j], w, wq, p)
                    assert t < 2 * p
                    x[i], x[j] = x[i] + t, x[i] - t + 2 * p
                    exact[i], exact[j] = (exact[i] + w * exact[j]) % p, (exact[i] - w * exact[j]) % p
                    top = max(top, x[i], x[j])
        assert top < 26 * p < 2 ** 31
        canon = [_lazy_mul(v, 1, one_q, p) for v in x]
        canon = [c - p if c >= p else c for c in canon]
        assert canon == exact
