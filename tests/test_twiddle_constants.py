"""The z convolution's compile-time twiddle constants (fields_ct.cu, cos_pi64:
cos(pi k / 64) for k = 0..32, written out to 21 digits) against the cosine,
read from the source so that a mistyped digit cannot pass: each entry must
round to the same double as cos(pi k / 64) computed here in 50-digit decimal
arithmetic (and agree with math.cos to an ulp)."""
import math
import os
import re
from decimal import Decimal, getcontext

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "magnum.af_b200", "csrc", "fields_ct.cu")


def _table():
    text = open(SRC).read()
    m = re.search(r"cos_pi64\(int k\) \{\s*constexpr double t\[33\] = \{(.*?)\};", text, re.S)
    assert m, "cos_pi64 table not found"
    return [Decimal(v.strip()) for v in m.group(1).split(",") if v.strip()]


def _cos(x):
    s, t, k = Decimal(0), Decimal(1), 0
    while abs(t) >= Decimal(10) ** -45:
        s += t
        k += 2
        t = -t * x * x / (k * (k - 1))
    return s


def test_cos_pi64_table():
    getcontext().prec = 50
    pi = Decimal("3.14159265358979323846264338327950288419716939937510")
    tab = _table()
    assert len(tab) == 33
    for k, v in enumerate(tab):
        exact = _cos(pi * k / 64) if k < 32 else Decimal(0)
        assert float(v) == float(exact), (k, v, exact)
        assert abs(float(v) - math.cos(math.pi * k / 64)) <= 2.3e-16, k
