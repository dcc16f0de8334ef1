#!/usr/bin/env python
"""Prints the 2^(j/128) table of nim_exp.cuh (NIM_EXP_TABLE_INIT).

For j = 0..127: H = 2^(j/128) rounded to the nearest double, T = the
relative error (2^(j/128) - H) / H rounded to the nearest double; the table
holds bits(T) and bits(H) - (j << 45), in that order.  2^(j/128) comes from
80-digit decimal arithmetic, far beyond double precision.
"""
import struct
from decimal import Decimal, getcontext


def bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def entries():
    getcontext().prec = 80
    out = []
    for j in range(128):
        exact = Decimal(2) ** (Decimal(j) / Decimal(128))
        h = float(exact)
        t = float((exact - Decimal(h)) / Decimal(h))
        out += [bits(t), (bits(h) - (j << 45)) % (1 << 64)]
    return out


if __name__ == "__main__":
    e = entries()
    for i in range(0, 256, 4):
        row = ", ".join(f"0x{v:016x}ULL" for v in e[i:i + 4])
        print(f"    {row}{',' if i < 252 else ''} \\")
