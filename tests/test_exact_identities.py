"""CPU checks of the exact substitutions the traversal kernel makes for the
reference's double-precision expressions (vfRayKernelCPU.cc), restated in
numpy: each substitution must give the reference's decision on every input
it accepts.

* exit-test slack (:341-342): (double)s <= (double)cr + 1e-12 for floats
  s, cr with cr >= 0x2b8cbccd  <=>  float(s - cr) <= 0x2b8cbccc;
* psi coordinate (:462-471): the float bracket around gamma = tau/(1.0+tau)
  selects the reference's table coordinate whenever its two ends agree, for
  any quotient estimate within the 2-ulp bound of __fdividef;
* keep = 1 - a of the compositing (:474-483) as zeta rounded to the 2^-24
  grid, for zeta in [0, 1];
* zeta's argument (:459) as one halved double sum.
"""
import numpy as np

F32 = np.float32
R = 1e-12
TH = np.array([0x2b8cbccc], np.uint32).view(F32)[0]  # largest float below 1e-12
CRMIN = np.array([0x2b8cbccd], np.uint32).view(F32)[0]


def test_slack_identity_near_the_threshold():
    rng = np.random.default_rng(7)
    bad = tot = 0
    for _ in range(8):
        cr = np.maximum((2.0 ** rng.uniform(-40, 20, 250_000)).astype(F32), CRMIN)
        ulp = np.spacing(cr).astype(np.float64)
        j0 = np.floor(R / ulp)
        for dj in (-2, -1, 0, 1, 2, 3):
            s = (cr.astype(np.float64) + np.maximum(j0 + dj, 0) * ulp).astype(F32)
            ref = s.astype(np.float64) <= cr.astype(np.float64) + R
            new = (s - cr) <= TH
            bad += int(np.count_nonzero(ref != new))
            tot += s.size
        s = (cr * rng.uniform(0.0, 3.0, cr.size)).astype(F32)
        ref = s.astype(np.float64) <= cr.astype(np.float64) + R
        bad += int(np.count_nonzero(ref != ((s - cr) <= TH)))
        tot += s.size
    assert tot > 10_000_000 and bad == 0


def _round_down(x64):
    """float32 rounding of float64 values toward -inf."""
    y = x64.astype(F32)
    hi = y.astype(np.float64) > x64
    y[hi] = np.nextafter(y[hi], F32(-np.inf))
    return y


def _round_up(x64):
    y = x64.astype(F32)
    lo = y.astype(np.float64) < x64
    y[lo] = np.nextafter(y[lo], F32(np.inf))
    return y


def _coord_ref(tau):
    """The reference: gamma in double, stored to float, + 0.5/512 in float."""
    t = tau.astype(np.float64)
    g = (t / (1.0 + t)).astype(F32)
    tc = (g.astype(np.float64) + 0.5 / 512).astype(F32)
    ok = (tc >= 0) & (tc <= 1)
    idx = np.minimum((tc * F32(512)).astype(np.uint32), 511)
    return np.where(ok, idx.astype(np.int64), -1)


def _floor512(t):
    # RD(t * 512 + 2^23) read back as an integer: floor(t * 512) for t in [0, 1]
    x = t.astype(np.float64) * 512.0 + 8388608.0
    return _round_down(x).view(np.uint32).astype(np.int64) - 0x4b000000


def test_psi_coordinate_bracket():
    rng = np.random.default_rng(11)
    tau = np.concatenate([(10.0 ** rng.uniform(-10, 6, 2_000_000)).astype(F32),
                          rng.uniform(0, 4, 1_000_000).astype(F32)])
    tau = tau[(tau > 0) & (tau < F32(1048576.0))]
    ref = _coord_ref(tau)
    d = (F32(1.0) + tau).astype(F32)
    q = (tau.astype(np.float64) / d.astype(np.float64)).astype(F32)
    accepted = 0
    for k in (-2, -1, 0, 1, 2):  # any estimate within 2 ulp of the float quotient
        g = q
        for _ in range(abs(k)):
            g = np.nextafter(g, F32(np.inf) if k > 0 else F32(-np.inf))
        tlo = ((_round_down(g.astype(np.float64) - 2.0 ** -20)).astype(np.float64) + 2.0 ** -10).astype(F32)
        thi = ((_round_up(g.astype(np.float64) + 2.0 ** -20)).astype(np.float64) + 2.0 ** -10).astype(F32)
        flo, fhi = _floor512(tlo), _floor512(thi)
        fast = (thi <= 1) & (flo == fhi)
        assert np.array_equal(np.minimum(flo[fast], 511), ref[fast])
        out = tlo > 1
        assert np.all(ref[out & ~fast] == -1)
        accepted += int(np.count_nonzero(fast | out))
    # the double division is needed for about one tau in a thousand
    assert accepted > 0.99 * 5 * tau.size


def test_division_through_a_shared_reciprocal():
    """float(RN_double(a * RN_double(1/b))) == a / b in float for every float
    quotient in the normal range: random pairs over many binades, and pairs
    built to put a / b next to a half-way point between floats."""
    rng = np.random.default_rng(5)
    n = 2_000_000
    b = (rng.choice([-1, 1], n) * 2.0 ** rng.uniform(-40, 4, n)).astype(F32)
    a = (rng.choice([-1, 1], n) * 2.0 ** rng.uniform(-60, 60, n)).astype(F32)
    # near half-way points: a = RN(M * 2^k * b) with M odd, 25 bits
    m = (rng.integers(1 << 24, 1 << 25, n) | 1).astype(np.float64)
    k = rng.integers(-50, 10, n).astype(np.float64)
    a2 = (m * 2.0 ** (k - 24) * b.astype(np.float64)).astype(F32)
    for num in (a, a2):
        with np.errstate(over="ignore", under="ignore"):
            want = num / b                                    # IEEE float division
            y = 1.0 / b.astype(np.float64)                    # correctly rounded reciprocal
            got = (num.astype(np.float64) * y).astype(F32)
        normal = np.abs(want) >= F32(2.0 ** -126)
        assert normal.mean() > 0.9
        assert np.array_equal(got[normal], want[normal])


def test_keep_is_zeta_on_the_2_pow_minus_24_grid():
    """keep = 1.0 - (double)(float)(1.0 - zeta) (:474-483) for a float zeta in
    [0, 1] is zeta rounded to a multiple of 2^-24, ties to even, which the
    kernel's fast path computes as (zeta + 1.5 * 2^28) - 1.5 * 2^28 in double.
    Checked on every float in [2^-27, 1] and on zero."""
    C = np.float64(1.5 * 2.0 ** 28)
    one = F32(1.0)
    for e in range(-27, 0):  # binade [2^e, 2^(e+1))
        lo = np.array([2.0 ** e], F32).view(np.uint32)[0]
        hi = np.array([2.0 ** (e + 1)], F32).view(np.uint32)[0]
        z = np.arange(lo, hi, dtype=np.uint32).view(F32)
        ref = 1.0 - (one - z).astype(np.float64)
        new = (z.astype(np.float64) + C) - C
        assert np.array_equal(ref.view(np.uint64), new.view(np.uint64)), e
    for z in (F32(0.0), F32(1.0), F32(2.0 ** -28), F32(1e-30)):
        z = np.array([z], F32)
        ref = 1.0 - (one - z).astype(np.float64)
        new = (z.astype(np.float64) + C) - C
        assert ref[0] == new[0]


def test_zeta_argument_as_one_halved_sum():
    """-(tau_f*0.5 + tau_b*0.5) in double (:459) equals (tau_f + tau_b) * -0.5
    for any floats: halving is exact and commutes with rounding, as no double
    sum of two floats is subnormal.  Bit for bit, signed zeros and infinities
    included."""
    rng = np.random.default_rng(11)
    for _ in range(4):
        n = 2_000_000
        a = (rng.uniform(0.5, 1.0, n) * 2.0 ** rng.integers(-149, 128, n)).astype(F32)
        b = (rng.uniform(0.5, 1.0, n) * 2.0 ** rng.integers(-149, 128, n)).astype(F32)
        near = rng.random(n) < 0.5  # half the pairs within a few binades of each other
        with np.errstate(over="ignore"):  # a few overflow to infinity, which stays exact
            b[near] = (a[near].astype(np.float64) * rng.uniform(0.01, 100, near.sum())).astype(F32)
        b[rng.random(n) < 0.01] = 0.0
        a64, b64 = a.astype(np.float64), b.astype(np.float64)
        ref = -((a64 * 0.5) + (b64 * 0.5))
        new = (a64 + b64) * -0.5
        assert np.array_equal(ref.view(np.uint64), new.view(np.uint64))
    z = np.zeros(1)
    assert (-((z * 0.5) + (z * 0.5))).view(np.uint64)[0] == ((z + z) * -0.5).view(np.uint64)[0]
