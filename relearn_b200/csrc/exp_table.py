"""Table of rl_exp (rl_math.cuh) and of the oracle's own_exp (oracle/shared_stream.h).

T_j = 2^(j/64) for j = 0..63 as a pair of doubles: hi = T_j rounded to nearest,
lo = (T_j - hi) rounded to nearest, from 60-digit decimal arithmetic.  Prints
the C initialiser both headers use (as exact hexadecimal literals):

    python relearn_b200/csrc/exp_table.py
"""
from decimal import Decimal, getcontext


def table(n: int = 64):
    getcontext().prec = 60
    out = []
    for j in range(n):
        t = Decimal(2) ** (Decimal(j) / Decimal(n))
        hi = float(t)
        lo = float(t - Decimal(hi))
        out.append((hi, lo))
    return out


def main():
    rows = table()
    print("{")
    for j, (hi, lo) in enumerate(rows):
        print(f"    {{ {hi.hex()}, {lo.hex()} }},  // 2^({j}/64)")
    print("}")


if __name__ == "__main__":
    main()
