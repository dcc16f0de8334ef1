"""The series constants of the float NIM coefficients (nim_direction_f32 in
csrc/nim_kernels.cuh) against the Bernoulli numbers: the function evaluates
h(x) = (x/(e^x-1) - 1 + x/2)/x^2 = sum_{n>=1} B_2n x^(2n-2)/(2n)! by Horner
in y = x^2 for |x| <= 2, so its constants must be B_2n/(2n)!, n = 1..8, and
the first term left out must be below 1e-8 of h there."""
import math
import re
from fractions import Fraction
from pathlib import Path

SRC = Path(__file__).resolve().parent.parent / "nim-conv22-shared_b200" / "csrc" / "nim_kernels.cuh"


def bernoulli(n_max: int):
    B = [Fraction(1)]
    for m in range(1, n_max + 1):
        B.append(-sum(math.comb(m + 1, j) * B[j] for j in range(m)) / Fraction(m + 1))
    return B


def horner_constants():
    text = SRC.read_text()
    body = text[text.index("void nim_direction_f32"):]
    body = body[:body.index("} else {")]
    first = re.search(r"float h = (-?)(\d+)\.f / (\d+)\.f;", body)
    rest = re.findall(r"h = fmaf\(h, y, (-?)(\d+)\.f / (\d+)\.f\);", body)
    consts = [first.groups()] + rest
    return [Fraction(int(a), int(b)) * (-1 if s else 1) for s, a, b in consts]


def test_constants_are_bernoulli_terms():
    B = bernoulli(20)
    want = [B[2 * n] / math.factorial(2 * n) for n in range(1, 9)]
    got = horner_constants()[::-1]          # Horner lists the highest power first
    assert got == want


def test_truncation_at_the_branch_point():
    B = bernoulli(20)
    y = Fraction(4)                          # |x| = 2
    h = sum(B[2 * n] / math.factorial(2 * n) * y ** (n - 1) for n in range(1, 9))
    first_left_out = abs(B[18] / math.factorial(18) * y ** 8)
    assert first_left_out / h < Fraction(1, 10 ** 8)
