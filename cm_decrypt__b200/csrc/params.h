// Parameter sets of the five Classic McEliece variants the reference decodes
// (CPU/param/param<set>/include/common.h:14-29; sk/ct byte counts from
// kem/variant_<set>/crypto_kem_mceliece<set>.h:4-6).  Shared by host and
// device code; the device kernels are templated on the set so every loop
// bound below is a compile-time constant there.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define CMD_HD __host__ __device__
#else
#define CMD_HD
#endif

namespace cmd {

enum : int { S348864 = 0, S460896 = 1, S6688128 = 2, S6960119 = 3, S8192128 = 4, NSETS = 5 };

template <int S> struct Set;

// Depth of the additive-FFT recursion for a degree-t locator: the smallest D
// with 2^D >= t + 1 (7 for t = 64, 96, 119; 8 for t = 128).
constexpr CMD_HD int fft_depth(int t)
{
    int d = 0;
    while ((1 << d) < t + 1)
        d++;
    return d;
}
// Depth of the transposed additive FFT that forms the 2t syndromes: the
// smallest D' with 2^D' >= 2t (7 for t = 64, 8 for t = 96, 119, 128; m - 5 for
// every set).
constexpr CMD_HD int synd_depth(int t) { return fft_depth(2 * t - 1); }
// M: GFBITS, N: SYS_N, T: SYS_T, CT: ciphertext = SYND_BYTES, SK: secret key.
#define CMD_DEFINE_SET(ID, ID_NUM, M_, N_, T_, CT_, SK_)                               \
    template <> struct Set<ID> {                                                       \
        static constexpr int id = ID_NUM, M = M_, N = N_, T = T_, CT = CT_, SK = SK_;  \
        static constexpr int SB = 8 * CT_;              /* bits fed to synd()   */     \
        static constexpr int MT = M_ * T_;              /* true syndrome bits   */     \
        static constexpr int NW = (N_ + 31) / 32;       /* error words per ct   */     \
        static constexpr int TW = T_;                   /* 2t u16 = t u32 words */     \
        static constexpr int TWP = (T_ + 3) / 4 * 4;    /* table row stride     */     \
        static constexpr int TWD = (2 * T_ * M_ + 127) / 128 * 4; /* dense row    */     \
        static constexpr int COND = (1 << (M_ - 4)) * (2 * M_ - 1);                    \
        static constexpr int CTW = (CT_ + 3) / 4;       /* ct as u32 words      */     \
    };
CMD_DEFINE_SET(S348864, 348864, 12, 3488, 64, 96, 6492)
CMD_DEFINE_SET(S460896, 460896, 13, 4608, 96, 156, 13608)
CMD_DEFINE_SET(S6688128, 6688128, 13, 6688, 128, 208, 13932)
CMD_DEFINE_SET(S6960119, 6960119, 13, 6960, 119, 194, 13948)
CMD_DEFINE_SET(S8192128, 8192128, 13, 8192, 128, 208, 14120)
#undef CMD_DEFINE_SET

struct SetInfo {
    int id, m, n, t, ct, sk, sb, nw, cond;
    CMD_HD int twp() const { return (t + 3) / 4 * 4; }  // syndrome-table row stride (words)
    CMD_HD int twd() const { return (2 * t * m + 127) / 128 * 4; }  // dense-table row stride (words)
};

CMD_HD inline SetInfo set_info(int s)
{
    switch (s) {
    case S348864: return {348864, 12, 3488, 64, 96, 6492, 768, 109, 5888};
    case S460896: return {460896, 13, 4608, 96, 156, 13608, 1248, 144, 12800};
    case S6688128: return {6688128, 13, 6688, 128, 208, 13932, 1664, 209, 12800};
    case S6960119: return {6960119, 13, 6960, 119, 194, 13948, 1552, 218, 12800};
    default: return {8192128, 13, 8192, 128, 208, 14120, 1664, 256, 12800};
    }
}

// Invokes f.template operator()<S>() with S the compile-time set index.
template <class F> inline auto dispatch_set(int s, F &&f)
{
    switch (s) {
    case S348864: return f.template operator()<S348864>();
    case S460896: return f.template operator()<S460896>();
    case S6688128: return f.template operator()<S6688128>();
    case S6960119: return f.template operator()<S6960119>();
    default: return f.template operator()<S8192128>();
    }
}

}  // namespace cmd
