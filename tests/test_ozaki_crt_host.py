"""Host logic of the modular (CRT) INT8 route, checked on the CPU against
Python big integers: the modulus table, the planner's exactness bounds and
the reconstruction step (the same code the device kernel runs, compiled for
the host)."""
import ctypes
import math

import numpy as np
import pytest


def _moduli(mf):
    return mf.ozaki_crt_moduli()


def test_moduli_pairwise_coprime_and_greedy(mf):
    mods = _moduli(mf)
    assert len(mods) == 49 and mods[0] == 256 and max(mods) <= 256
    for i, p in enumerate(mods):
        for q in mods[:i]:
            assert math.gcd(p, q) == 1, (p, q)
    # greedy: every skipped number between consecutive entries shares a factor
    chosen = []
    for p in range(256, 1, -1):
        if all(math.gcd(p, q) == 1 for q in chosen):
            chosen.append(p)
    assert chosen == mods


def _P(mods, T):
    P = 1
    for p in mods[:T]:
        P *= p
    return P


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("k", [1, 100, 2048, 8192, 30000])
def test_plan_keeps_level_sums_exact(mf, N, k):
    """for every modulus count the digit width keeps every level sum within
    3P / 8 (one digit: |D| <= 2^(h-1) + 2^(h-52) + 2 from the (-1/2, 1/2)
    scaling, the lower limbs and the limb rounding; two digits: 2^(h+1), up
    to 2 kp terms per level) and the int32 sums exact"""
    mods = _moduli(mf)
    kp = max(128, (k + 127) // 128 * 128)
    for T in range(20, 50):
        try:
            plan = mf.ozaki_crt_plan(N, k, moduli=T)
        except (mf.MFLABError, mf.ArgumentError):
            continue
        Q, h = plan["digits"], plan["digit_bits"]
        assert plan["moduli"] == T and Q == (1 if N == 2 else 2)
        # every level sum stays within 3P / 8, the reconstruction's range
        if Q == 1:
            bound = 2 ** (h - 1) + 2 ** (h - 52) + 2
            assert 8 * kp * bound * bound <= 3 * _P(mods, T)
        else:
            bound = 2 ** (h + 1)
            assert 8 * Q * kp * bound * bound <= 3 * _P(mods, T)
        assert Q * kp * 2 ** 14 < 2 ** 31


@pytest.mark.parametrize("N", [2, 3, 4])
@pytest.mark.parametrize("gap", [0.0, 7.5, 20.0, 33.0])
def test_tuner_reaches_required_bits(mf, N, gap):
    """the tuned plan carries at least 53 N + 1 + gap + 7 bits below the
    row/column scale, with the fewest moduli that allow it"""
    k = 4096
    plan = mf.ozaki_crt_plan(N, k, 0, gap)
    Q, h, T = plan["digits"], plan["digit_bits"], plan["moduli"]
    need = math.ceil(53 * N + 1 + gap + 7)
    assert Q * h >= need + (Q - 1)
    if T > 1:
        smaller = mf.ozaki_crt_plan(N, k, moduli=T - 1)
        assert smaller["digit_bits"] < h


def test_plan_rejects_out_of_table(mf):
    with pytest.raises(mf.ArgumentError):
        mf.ozaki_crt_plan(2, 4096, 0, 200.0)  # needs more than 49 moduli
    with pytest.raises(mf.ArgumentError):
        mf.ozaki_crt_plan(4, 70000, moduli=40)  # Q kp 2^14 >= 2^31


def _reduce(mf, T, G):
    lib = mf._native.load()
    G = np.ascontiguousarray(G, dtype=np.int32)
    cnt = G.shape[0]
    mag = np.zeros((cnt, 12), dtype=np.uint32)
    neg = np.zeros(cnt, dtype=np.int32)
    rc = lib.mflab_ozaki_crt_reduce_host(T, cnt, G.ctypes.data, mag.ctypes.data, neg.ctypes.data)
    assert rc == 0
    out = []
    for e in range(cnt):
        v = sum(int(mag[e, w]) << (32 * w) for w in range(12))
        out.append(-v if neg[e] else v)
    return out


@pytest.mark.parametrize("T", [2, 3, 17, 32, 33, 40, 49])
def test_crt_reconstruction_matches_bigint(mf, T):
    mods = _moduli(mf)
    P = _P(mods, T)
    rng = np.random.default_rng(T)
    # inside the reconstruction's range |x| <= 3P / 8 (the planner keeps every
    # level sum there), including P / 4
    xs = [0, 1, -1, P // 4, -(P // 4)]
    for _ in range(200):
        bits = int(rng.integers(1, P.bit_length()))
        v = int.from_bytes(rng.bytes(64), "little") % (1 << bits)
        v %= P // 4 + 1
        xs.append(v if rng.random() < 0.5 else -v)
    G = np.zeros((len(xs), T), dtype=np.int64)
    for e, x in enumerate(xs):
        for t, p in enumerate(mods[:T]):
            r = x % p
            # any int32 representative, as an int8 GEMM would produce it
            r += p * int(rng.integers(-(2 ** 31 - 256) // p, (2 ** 31 - 256) // p))
            G[e, t] = r
    got = _reduce(mf, T, G)
    assert got == xs


def test_crt_reconstruction_of_int8_products(mf):
    """residues of an exact integer dot product, formed as the GEMM forms them
    (signed-byte residues of each factor, int32 sum), reconstruct the product"""
    mods = _moduli(mf)
    T = 33
    rng = np.random.default_rng(7)
    k = 300
    a = [int.from_bytes(rng.bytes(14), "little") - (1 << 111) for _ in range(k)]
    b = [int.from_bytes(rng.bytes(14), "little") - (1 << 111) for _ in range(k)]
    exact = sum(x * y for x, y in zip(a, b))
    assert abs(exact) < _P(mods, T) // 2

    def sres(x, p):
        r = x % p
        return r - p if r >= 128 else r

    G = np.zeros((1, T), dtype=np.int64)
    for t, p in enumerate(mods[:T]):
        G[0, t] = sum(sres(x, p) * sres(y, p) for x, y in zip(a, b))
        assert abs(G[0, t]) < 2 ** 31
    assert _reduce(mf, T, G) == [exact]


def test_scheme_selection(mf):
    K = mf.KernelConfig
    assert mf.ozaki_scheme(K()) == "modular"
    assert mf.ozaki_scheme(K(ozaki_slices=12)) == "slices"
    assert mf.ozaki_scheme(K(ozaki_scheme="slices")) == "slices"
    assert mf.ozaki_scheme(K(ozaki_scheme="modular", ozaki_moduli=30)) == "modular"
    with pytest.raises(mf.ArgumentError):
        mf.ozaki_scheme(K(ozaki_scheme="bogus"))
