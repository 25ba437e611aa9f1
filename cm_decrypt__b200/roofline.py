"""Algorithmic work per decryption: the int-ALU roofline of the decrypt kernels.

A GF(2^m) multiply is counted as m^2 fused AND-XOR bit operations plus R_m
reduction XORs (R_12 = 22 for the trinomial x^12+x^3+1, R_13 = 48 for the
pentanomial x^13+x^4+x^3+x+1); one 32-bit lop3 performs 32 bit operations,
so every figure below is bit operations / 32 ("lane-ops").

Work of the algorithm the fused kernel executes, per decryption:

  W_synd = (sb / 4) * (NWU + 11 * NWU / R)
           the dense table in groups of four rows: the CTA forms the group's
           16 XOR combinations (11 word XORs per accumulator word, shared by
           the R ciphertexts of a full round: 32 per warp of the CTA), and
           each ciphertext adds the one its four bits select
           (NWU = ceil(2tm / 32) words)
  W_bm   = [sum_{N<2t} (min(N, t, L_N) + 1) + 2 sum_{N<2t} (min(L_{N+1}, t) + 1)]
           * (m^2 + R_m) / 32
           (the scaled, L-bounded Berlekamp-Massey: discrepancy terms up to
           the current L, then b*C_i + d*B_i for the coefficients up to the
           new L; L_N = floor((N+1)/2), the trajectory of a weight-t error)
  W_root = additive FFT at all 2^m field elements, D = ceil(log2(t+1)):
           [ (D-1) 2^D (m^2+R_m)                   radix-conversion scalings
           + 2^(D-2) m D(D-1)                      Taylor-expansion XORs
           + D 2^(m-1) (m^2 + R_m + 2m)            butterflies
           + 2^m m                                 zero flags
           + (2m-1) 2^(m-1) 3 ] / 32               support network swaps

``achieved = decaps/s * (W_synd + W_bm + W_root)`` lane-ops/s against the
measured lop3 rate.

The fixed yardstick of the reference's algorithm is kept beside it, as the
work table of the decrypt path's scope defines it:

  W_synd_table = sb * 2t * m / 32            masked XOR of every set bit's row
  W_bm_ref     = [sum_{N<2t} (min(N,t) + 1) + 2t(t+1) + 8 * 2t] * (m^2 + R_m) / 32
                 (bm()'s discrepancy and update multiplies, each step's d/b as
                 eight multiply-equivalents)
  W_chien      = n * t * (m^2 + R_m + m) / 32   Horner at every support point
                 (root_13.c:216-240)

The plain per-stage kernels, which run the reference's algorithm, are
measured against those three, stage by stage.

Bytes per decryption that must cross HBM: the ciphertext in and the n-bit
error vector out.
"""
from __future__ import annotations

SETS = {348864: (12, 3488, 64, 96), 460896: (13, 4608, 96, 156), 6688128: (13, 6688, 128, 208),
        6960119: (13, 6960, 119, 194), 8192128: (13, 8192, 128, 208)}
ROUND_CTS = 256  # ciphertexts sharing one CTA's combinations: 8 warps of 32


def fft_depth(t: int) -> int:
    d = 0
    while (1 << d) < t + 1:
        d += 1
    return d


def work_per_decap(set_id: int, round_cts: int = ROUND_CTS) -> dict:
    m, n, t, ct = SETS[set_id]
    r = 22 if m == 12 else 48
    mul = m * m + r
    sb = 8 * ct
    nwu = (2 * t * m + 31) // 32
    w_synd = sb / 4 * (nwu + 11 * nwu / round_cts)
    disc = sum(min(N, t, (N + 1) // 2) + 1 for N in range(2 * t))
    upd = sum(min((N + 2) // 2, t) + 1 for N in range(2 * t))
    w_bm = (disc + 2 * upd) * mul / 32
    D = fft_depth(t)
    w_root = ((D - 1) * (1 << D) * mul + (1 << (D - 2)) * m * D * (D - 1)
              + D * (1 << (m - 1)) * (mul + 2 * m) + (1 << m) * m + (2 * m - 1) * (1 << (m - 1)) * 3) / 32
    ys = sb * 2 * t * m / 32
    yb = (sum(min(N, t) + 1 for N in range(2 * t)) + 2 * t * (t + 1) + 16 * t) * mul / 32
    yc = n * t * (mul + m) / 32
    return {"synd": w_synd, "bm": w_bm, "root_fft": w_root, "total": w_synd + w_bm + w_root,
            "yardstick_synd_table": ys, "yardstick_bm_ref": yb, "yardstick_chien": yc,
            "yardstick_total": ys + yb + yc}


def plain_stage_work(set_id: int) -> dict:
    """Lane-ops per decryption of the reference algorithm of each plain stage."""
    w = work_per_decap(set_id)
    return {"synd": w["yardstick_synd_table"], "bm": w["yardstick_bm_ref"], "root": w["yardstick_chien"]}


def hbm_bytes_per_decap(set_id: int) -> int:
    m, n, t, ct = SETS[set_id]
    return ct + n // 8
