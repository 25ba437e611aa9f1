"""Algorithmic work per decryption, the fixed yardstick for the int-ALU
roofline of the decrypt kernels.

A GF(2^m) multiply is counted as m^2 fused AND-XOR bit operations plus R_m
reduction XORs (R_12 = 22 for the trinomial x^12+x^3+1, R_13 = 48 for the
pentanomial x^13+x^4+x^3+x+1); one 32-bit lop3 performs 32 bit operations.
Per decryption:

  W_synd  = sb * 2t * m / 32                     masked XOR of table rows
  W_bm    = [sum_{N<2t} (min(N,t)+1) + 2t(t+1) + 8*2t] * (m^2 + R_m) / 32
            (discrepancies, C updates, d/b counted as 8 multiplies)
  W_chien = n * t * (m^2 + R_m + m) / 32          Horner at every support point

so ``achieved = decaps/s * W`` lane-ops/s, compared with the measured lop3
rate.  A root finder that does less work than Horner still divides by the
same W.  Bytes per decryption that must cross HBM: the ciphertext in and the
n-bit error vector out.
"""
from __future__ import annotations

SETS = {348864: (12, 3488, 64, 96), 460896: (13, 4608, 96, 156), 6688128: (13, 6688, 128, 208),
        6960119: (13, 6960, 119, 194), 8192128: (13, 8192, 128, 208)}


def work_per_decap(set_id: int) -> dict:
    m, n, t, ct = SETS[set_id]
    r = 22 if m == 12 else 48
    sb = 8 * ct
    w_synd = sb * 2 * t * m / 32
    disc = sum(min(N, t) + 1 for N in range(2 * t))
    w_bm = (disc + 2 * t * (t + 1) + 8 * 2 * t) * (m * m + r) / 32
    w_chien = n * t * (m * m + r + m) / 32
    return {"synd": w_synd, "bm": w_bm, "chien": w_chien, "total": w_synd + w_bm + w_chien}


def hbm_bytes_per_decap(set_id: int) -> int:
    m, n, t, ct = SETS[set_id]
    return ct + n // 8
