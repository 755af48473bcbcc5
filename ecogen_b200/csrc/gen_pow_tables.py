"""Writes ecg_pow_tables.h, the tables of the table-driven pow of ecg_pow.cuh.

Run from this folder: python gen_pow_tables.py (needs mpmath; the generated header is committed, so a
build does not run this).  Every entry is computed with 200-bit arithmetic and rounded to nearest:

* log table, 128 rows, one per subinterval [1 + i/128, 1 + (i+1)/128) of the significand m:
  inv_i ~ 1 / (the subinterval's centre) rounded to a multiple of 2^-8 (row 0: inv = 1), so that
  r = m inv_i - 1 is exact in one FMA (|r| < 2^-7 and m inv_i is a multiple of 2^-60), and
  -ln(inv_i) as a double-double (hi, lo), except row 127 (inv = 1/2), which holds the split L2H + L2L
  of ln 2 below;
* exp table, 128 rows: 2^(j/128) as a double-double (hi, lo);
* ln 2 split as L2H (40 significant bits, so k * L2H is exact for |k| < 2^12) + L2L; ln 2 / 128 split
  as C1 + C2 (C1 = RN(ln 2 / 128), whose last bit is 2^-60, so Y - kd C1 is exact for |kd| < 2^12);
  INVC = RN(128 / ln 2).
"""
import os

import mpmath as mp

mp.mp.prec = 200
N = 128


def dd(v):
    hi = float(v)
    return hi, float(v - mp.mpf(hi))


def main():
    log_rows, max_r = [], mp.mpf(0)
    for i in range(N):
        inv = mp.mpf(1) if i == 0 else mp.nint(256 / (1 + (mp.mpf(i) + mp.mpf("0.5")) / N)) / 256
        for m in (1 + mp.mpf(i) / N, 1 + mp.mpf(i + 1) / N):
            max_r = max(max_r, abs(m * inv - 1))
        hi, lo = dd(-mp.log(inv))
        log_rows.append((float(inv), hi, lo))
    # row 127 (inv = 1/2): -ln(1/2) = ln 2, stored with the split of k ln 2 so that for x just below 1
    # (k = -1) the two cancel exactly and ln x = ln(1 + r)
    ln2 = mp.log(2)
    l2h = float(mp.floor(ln2 * 2 ** 40) / 2 ** 40)
    l2l = float(ln2 - mp.mpf(l2h))
    assert log_rows[127][0] == 0.5
    log_rows[127] = (0.5, l2h, l2l)
    assert max_r <= mp.mpf(2) ** -7, "r must stay below 2^-7 for m inv - 1 to be exact"
    exp_rows = [dd(mp.power(2, mp.mpf(j) / N)) for j in range(N)]
    c1 = float(ln2 / N)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ecg_pow_tables.h")
    with open(out, "w") as f:
        f.write("// Generated by gen_pow_tables.py (200-bit arithmetic, rounded to nearest); see ecg_pow.cuh.\n")
        f.write("#pragma once\n\n")
        f.write("// {inv_i, -ln(inv_i) hi, lo} for significands in [1 + i/128, 1 + (i+1)/128)\n")
        f.write("ECG_POW_TABLE double ecg_pow_logt[128][3] = {\n")
        for inv, hi, lo in log_rows:
            f.write(f"    {{{inv.hex()}, {hi.hex()}, {lo.hex()}}},\n")
        f.write("};\n// {2^(j/128) hi, lo}\n")
        f.write("ECG_POW_TABLE double ecg_pow_expt[128][2] = {\n")
        for hi, lo in exp_rows:
            f.write(f"    {{{hi.hex()}, {lo.hex()}}},\n")
        f.write("};\n")
        f.write(f"constexpr double ECG_POW_L2H = {l2h.hex()}, ECG_POW_L2L = {l2l.hex()};\n")
        f.write(f"constexpr double ECG_POW_C1 = {c1.hex()}, ECG_POW_C2 = {float(ln2 / N - mp.mpf(c1)).hex()};\n")
        f.write(f"constexpr double ECG_POW_INVC = {float(N / ln2).hex()};\n")
    print("wrote", out, "max |r| = 2^%.3f" % float(mp.log(max_r, 2)))


if __name__ == "__main__":
    main()
