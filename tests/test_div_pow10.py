"""The DECIMAL → float64 conversion divides by math.Pow10(scale) without a
division instruction (wg_device.cuh: div_pow10, Markstein's correction with a
table of reciprocals). This checks, on the CPU and in exact rational
arithmetic, that the table holds RN(1/Pow10(n)) and that the device's sequence
of one multiply and four fused multiply-adds returns the correctly rounded
quotient, which is what Go's `/` (Int128.ToFloat64, decimal.go:39-51) gives."""
import os
import random
import re
from fractions import Fraction

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "wadjet_b200", "csrc")


def pow10_go(n: int) -> float:
    """math.Pow10 for 0 <= n < 128: pow10tab[n%32] * pow10postab32[n/32], one rounding."""
    return float("1e%d" % (n % 32)) * [1e0, 1e32, 1e64, 1e96][n // 32]


def recip_table() -> list[float]:
    src = open(os.path.join(CSRC, "wg_device.cuh")).read()
    body = re.search(r"#define WG_POW10_RECIP \\\n(.*?)\nstatic __constant__ double c_pow10_recip", src, re.S).group(1)
    return [float.fromhex(x) for x in re.findall(r"0x[0-9a-fA-Fp.+-]+", body)]


def fma(x: float, y: float, z: float) -> float:
    return float(Fraction(x) * Fraction(y) + Fraction(z))  # int/int true division rounds correctly


def div_pow10(a: float, n: int, y: list[float]) -> float:
    if n <= 0 or n >= 128:
        return a
    b = pow10_go(n)
    q = a * y[n]
    r = fma(-q, b, a)
    q = fma(r, y[n], q)
    r = fma(-q, b, a)
    return fma(r, y[n], q)


def test_reciprocal_table_is_correctly_rounded():
    y = recip_table()
    assert len(y) == 128
    for n in range(128):
        assert y[n] == float(Fraction(1) / Fraction(pow10_go(n))), n


def test_division_is_correctly_rounded():
    y = recip_table()
    rng = random.Random(7)
    cases = [(float(v), n) for v in (1, -1, 5, 25, 125, 2**53 - 1, 2**53 + 2, 2**63 - 1, -(2**63))
             for n in range(40)]
    for _ in range(20_000):
        bits = rng.choice([8, 17, 32, 47, 53, 54, 63, 64, 90, 127])
        v = rng.getrandbits(bits) or 1
        cases.append((float(v if rng.random() < 0.5 else -v), rng.choice(range(128)) if rng.random() < 0.2
                      else rng.randrange(39)))
    for a, n in cases:
        want = float(Fraction(a) / Fraction(pow10_go(n))) if 0 < n < 128 else a
        assert div_pow10(a, n, y) == want, (a, n)
