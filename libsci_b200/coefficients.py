"""Derivation of the polynomial in sci_math.cuh's tanh_float_near (float tanh for |x| <= 1).

tanh x = x + x^3 g(x^2), g(u) = (tanh(sqrt u) / sqrt u - 1) / u, smooth on [0, 1] (g(0) = -1/3).
The coefficients are those of the degree-11 polynomial interpolating g at the 12 Chebyshev nodes
of [0, 1], solved in 60-digit decimal arithmetic and rounded to double. The script prints them
(lowest degree first, as C hex floats) and the largest relative error of the rounded polynomial
against g on 20001 evenly spaced points of [0, 1], evaluated in the same arithmetic.

Usage: python -m libsci_b200.coefficients
"""
from __future__ import annotations

import math
from decimal import Decimal, getcontext

getcontext().prec = 60
DEGREE = 11
PI = Decimal("3.14159265358979323846264338327950288419716939937510582097494")


def tanh(a: Decimal) -> Decimal:
    e = (2 * a).exp()
    return (e - 1) / (e + 1)


def g(u: Decimal) -> Decimal:
    if u == 0:
        return Decimal(-1) / 3
    a = u.sqrt()
    return (tanh(a) / a - 1) / u


def cos(x: Decimal) -> Decimal:
    total, term, k = Decimal(1), Decimal(1), 0
    while True:
        k += 2
        term = -term * x * x / (k * (k - 1))
        if abs(term) < Decimal(10) ** -58:
            return total
        total += term


def solve(matrix, right):
    """Gaussian elimination with partial pivoting, in Decimal."""
    n = len(right)
    rows = [list(row) + [right[i]] for i, row in enumerate(matrix)]
    for i in range(n):
        pivot = max(range(i, n), key=lambda r: abs(rows[r][i]))
        rows[i], rows[pivot] = rows[pivot], rows[i]
        for r in range(i + 1, n):
            f = rows[r][i] / rows[i][i]
            for c in range(i, n + 1):
                rows[r][c] -= f * rows[i][c]
    x = [Decimal(0)] * n
    for i in reversed(range(n)):
        x[i] = (rows[i][n] - sum(rows[i][c] * x[c] for c in range(i + 1, n))) / rows[i][i]
    return x


def coefficients(degree: int = DEGREE) -> list[float]:
    m = degree + 1
    nodes = [Decimal(1) / 2 + cos((2 * i + 1) * PI / (2 * m)) / 2 for i in range(m)]
    exact = solve([[x ** j for j in range(m)] for x in nodes], [g(x) for x in nodes])
    return [float(c) for c in exact]


def worst_relative_error(coefs: list[float], points: int = 20001) -> float:
    worst = Decimal(0)
    for i in range(points):
        u = Decimal(i) / (points - 1)
        value = Decimal(0)
        for c in reversed(coefs):
            value = value * u + Decimal(c)
        worst = max(worst, abs((value - g(u)) / g(u)))
    return float(worst)


if __name__ == "__main__":
    coefs = coefficients()
    error = worst_relative_error(coefs)
    print(f"degree {DEGREE}: relative error {error:.3e} = 2^{math.log2(error):.2f}")
    for c in coefs:
        print(c.hex())
