// Synthetic workloads: seeded secret keys and ciphertexts for any of the five
// parameter sets, so batches of 2^20 fresh ciphertexts per set can be made on
// the host without the reference's kem/ generator (whose third-party AES and
// Keccak code is not shipped).
//
// Keys are derived from a base key of the same set: its Goppa polynomial g is
// translated, g(y) -> g(y + c) (a ring automorphism, so irreducibility and
// monicity are kept), and the Benes control bits are drawn fresh; any
// control-bit setting of a Benes network is a permutation, so the support
// stays a list of distinct field elements.  A draw is kept only if the first
// mt support columns of the parity-check matrix are invertible (the
// systematic-form condition the reference keygen also enforces).
//
// Ciphertexts are Niederreiter syndromes c = [I | X] e for the systematic
// parity-check matrix, e of weight exactly t with positions uniform over
// [0, n); malformed ones are uniform mt-bit strings.  Decoding a valid one
// must flag exactly the positions of e.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "cmd_b200.h"
#include "params.h"

namespace {

using cmd::SetInfo;

// ---- seeded generator: SplitMix64 (Steele, Lea, Flood 2014) ------------
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint32_t below(uint32_t n) { return (uint32_t)(((unsigned __int128)next() * n) >> 64); }
};
static uint64_t mix(uint64_t a, uint64_t b) { return Rng(a ^ Rng(b).next()).next(); }

// ---- host field arithmetic ----------------------------------------------
struct Field {
    int m;
    uint32_t poly;
    explicit Field(int m_) : m(m_), poly(m_ == 12 ? 0x1009u : 0x201Bu) {}
    uint16_t mul(uint32_t a, uint32_t b) const
    {
        uint32_t p = 0;
        for (int i = 0; i < m; i++)
            if ((b >> i) & 1u)
                p ^= a << i;
        for (int k = 2 * m - 2; k >= m; k--)
            if ((p >> k) & 1u)
                p ^= poly << (k - m);
        return (uint16_t)p;
    }
    uint16_t inv(uint32_t a) const
    {
        uint32_t e = (1u << m) - 2u, r = 1, b = a;
        while (e) {
            if (e & 1u)
                r = mul(r, b);
            b = mul(b, b);
            e >>= 1;
        }
        return (uint16_t)r;
    }
};

static uint16_t load_coeff(const uint8_t *p, int m) { return (uint16_t)((p[0] | (p[1] << 8)) & ((1u << m) - 1u)); }

// Support from Benes control bits: the element-wise statement of the network
// (layer l exchanges p, p + 2^e when control bit l*2^(m-1) + (p without bit e)
// is set; e = l, then 2m-2-l), applied to bitrev(0..2^m-1).
static void support_from_cond(const SetInfo &si, const uint8_t *cond, std::vector<uint16_t> &L)
{
    const int m = si.m;
    const uint32_t size = 1u << m, half = size / 2;
    std::vector<uint16_t> v(size);
    for (uint32_t i = 0; i < size; i++) {
        uint32_t r = 0;
        for (int b = 0; b < m; b++)
            if ((i >> b) & 1u)
                r |= 1u << (m - 1 - b);
        v[i] = (uint16_t)r;
    }
    for (int layer = 0; layer < 2 * m - 1; layer++) {
        const int e = layer < m ? layer : 2 * m - 2 - layer;
        for (uint32_t q = 0; q < half; q++) {
            const uint32_t p = ((q >> e) << (e + 1)) | (q & ((1u << e) - 1u));
            const uint32_t bit = (uint32_t)layer * half + q;
            if ((cond[bit >> 3] >> (bit & 7)) & 1u)
                std::swap(v[p], v[p + (1u << e)]);
        }
    }
    L.assign(v.begin(), v.begin() + si.n);
}

// Parity-check rows r = j*m + k (j < t, k < m): bit i = bit k of L_i^j / g(L_i).
// Row-major bitsets over `cols` columns.
struct BitMatrix {
    int rows = 0, cols = 0, words = 0;
    std::vector<uint64_t> d;
    void init(int r, int c)
    {
        rows = r;
        cols = c;
        words = (c + 63) / 64;
        d.assign((size_t)r * words, 0);
    }
    uint64_t *row(int r) { return d.data() + (size_t)r * words; }
};

static void parity_check(const SetInfo &si, const Field &F, const std::vector<uint16_t> &g,
                         const std::vector<uint16_t> &L, int cols, BitMatrix &H)
{
    const int m = si.m, t = si.t;
    H.init(m * t, cols);
    for (int i = 0; i < cols; i++) {
        uint32_t v = g[t];
        for (int j = t - 1; j >= 0; j--)
            v = F.mul(v, L[i]) ^ g[j];
        uint32_t x = F.inv(v);
        for (int j = 0; j < t; j++) {
            for (int k = 0; k < m; k++)
                if ((x >> k) & 1u)
                    H.row(j * m + k)[i >> 6] |= 1ull << (i & 63);
            x = F.mul(x, L[i]);
        }
    }
}

// Gauss-Jordan on the first mt columns; false if that block is singular.
static bool systematize(BitMatrix &H, int mt)
{
    for (int c = 0; c < mt; c++) {
        const int w = c >> 6;
        const uint64_t bit = 1ull << (c & 63);
        int p = c;
        while (p < H.rows && !(H.row(p)[w] & bit))
            p++;
        if (p == H.rows)
            return false;
        if (p != c)
            std::swap_ranges(H.row(p), H.row(p) + H.words, H.row(c));
        const uint64_t *pr = H.row(c);
        for (int r = 0; r < H.rows; r++) {
            if (r == c || !(H.row(r)[w] & bit))
                continue;
            uint64_t *rr = H.row(r);
            for (int q = w; q < H.words; q++)
                rr[q] ^= pr[q];
        }
    }
    return true;
}

static void goppa_from_sk(const SetInfo &si, const uint8_t *sk, std::vector<uint16_t> &g)
{
    g.resize(si.t + 1);
    for (int i = 0; i < si.t; i++)
        g[i] = load_coeff(sk + 40 + 2 * i, si.m);
    g[si.t] = 1;
}

// g(y + c): coefficients of the Taylor shift by repeated synthetic division.
static std::vector<uint16_t> translate(const Field &F, std::vector<uint16_t> g, uint16_t c)
{
    const int t = (int)g.size() - 1;
    for (int i = 0; i < t; i++)
        for (int j = t - 1; j >= i; j--)
            g[j] ^= F.mul(g[j + 1], c);
    return g;
}

}  // namespace

struct cmd_pubkey {
    SetInfo si;
    int mt = 0, xwords = 0;
    std::vector<uint64_t> xcols;  // column i >= mt of X, xwords words each
};

extern "C" {

int cmd_synth_key(cmd_set set, const uint8_t *h_base_sk, uint64_t seed, uint8_t *h_sk_out)
{
    if (set < 0 || set >= cmd::NSETS || !h_base_sk || !h_sk_out)
        return CMD_E_ARG;
    const SetInfo si = cmd::set_info(set);
    const Field F(si.m);
    std::vector<uint16_t> g;
    goppa_from_sk(si, h_base_sk, g);
    Rng rng(mix(seed, 0x6b6579ull + (uint64_t)si.id));
    g = translate(F, g, (uint16_t)rng.below(1u << si.m));
    std::vector<uint8_t> sk(h_base_sk, h_base_sk + si.sk);
    for (int i = 0; i < si.t; i++) {
        sk[40 + 2 * i] = (uint8_t)(g[i] & 0xFF);
        sk[41 + 2 * i] = (uint8_t)(g[i] >> 8);
    }
    const int mt = si.m * si.t;
    uint8_t *cond = sk.data() + 40 + 2 * si.t;
    for (int attempt = 0; attempt < 256; attempt++) {
        for (int b = 0; b < si.cond; b++)
            cond[b] = (uint8_t)rng.next();
        std::vector<uint16_t> L;
        support_from_cond(si, cond, L);
        BitMatrix H;
        parity_check(si, F, g, L, mt, H);
        if (systematize(H, mt)) {
            uint8_t *s = sk.data() + 40 + 2 * si.t + si.cond;
            for (int b = 0; b < si.n / 8; b++)
                s[b] = (uint8_t)rng.next();
            memcpy(h_sk_out, sk.data(), si.sk);
            return CMD_OK;
        }
    }
    return CMD_E_ARG;
}

int cmd_synth_pubkey(cmd_set set, const uint8_t *h_sk, cmd_pubkey **out)
{
    if (set < 0 || set >= cmd::NSETS || !h_sk || !out)
        return CMD_E_ARG;
    *out = nullptr;
    const SetInfo si = cmd::set_info(set);
    const Field F(si.m);
    std::vector<uint16_t> g, L;
    goppa_from_sk(si, h_sk, g);
    support_from_cond(si, h_sk + 40 + 2 * si.t, L);
    const int mt = si.m * si.t;
    BitMatrix H;
    parity_check(si, F, g, L, si.n, H);
    if (!systematize(H, mt))
        return CMD_E_ARG;
    std::unique_ptr<cmd_pubkey> pk(new cmd_pubkey());
    pk->si = si;
    pk->mt = mt;
    pk->xwords = (mt + 63) / 64;
    pk->xcols.assign((size_t)(si.n - mt) * pk->xwords, 0);
    for (int r = 0; r < mt; r++) {
        const uint64_t *row = H.row(r);
        for (int i = mt; i < si.n; i++)
            if ((row[i >> 6] >> (i & 63)) & 1u)
                pk->xcols[(size_t)(i - mt) * pk->xwords + (r >> 6)] |= 1ull << (r & 63);
    }
    *out = pk.release();
    return CMD_OK;
}

void cmd_synth_pubkey_free(cmd_pubkey *pk) { delete pk; }

int cmd_pubkey_columns(const cmd_pubkey *pk, uint64_t *out, size_t cap_words, size_t *words_per_col)
{
    if (!pk || !words_per_col)
        return CMD_E_ARG;
    *words_per_col = (size_t)pk->xwords;
    if (!out)
        return CMD_OK;
    if (cap_words < pk->xcols.size())
        return CMD_E_ARG;
    memcpy(out, pk->xcols.data(), pk->xcols.size() * sizeof(uint64_t));
    return CMD_OK;
}

int cmd_synth_ciphertexts(const cmd_pubkey *pk, uint64_t seed, size_t count, uint32_t malformed_permille,
                          uint8_t *h_cts_out, uint8_t *h_err_out, uint8_t *h_valid_out, int nthreads)
{
    if (!pk || (count && !h_cts_out) || malformed_permille > 1000)
        return CMD_E_ARG;
    const SetInfo si = pk->si;
    const int mt = pk->mt, xw = pk->xwords;
    auto work = [&](size_t begin, size_t end) {
        std::vector<uint64_t> c(xw);
        std::vector<uint8_t> used(si.n);
        std::vector<uint16_t> pos(si.t);
        for (size_t i = begin; i < end; i++) {
            Rng rng(mix(seed, i));
            uint8_t *ct = h_cts_out + i * si.ct;
            uint8_t *ev = h_err_out ? h_err_out + i * (si.n / 8) : nullptr;
            const bool bad = rng.below(1000) < malformed_permille;
            if (h_valid_out)
                h_valid_out[i] = bad ? 0 : 1;
            if (ev)
                memset(ev, 0, si.n / 8);
            std::fill(c.begin(), c.end(), 0);
            if (bad) {
                for (int w = 0; w < xw; w++)
                    c[w] = rng.next();
            } else {
                int got = 0;
                while (got < si.t) {
                    const uint32_t p = rng.below(si.n);
                    if (used[p])
                        continue;
                    used[p] = 1;
                    pos[got++] = (uint16_t)p;
                }
                for (int k = 0; k < si.t; k++) {
                    const int p = pos[k];
                    used[p] = 0;
                    if (ev)
                        ev[p >> 3] |= (uint8_t)(1u << (p & 7));
                    if (p < mt) {
                        c[p >> 6] ^= 1ull << (p & 63);
                    } else {
                        const uint64_t *col = pk->xcols.data() + (size_t)(p - mt) * xw;
                        for (int w = 0; w < xw; w++)
                            c[w] ^= col[w];
                    }
                }
            }
            if (mt % 64)
                c[xw - 1] &= (1ull << (mt % 64)) - 1;  // padding bits stay zero
            for (int b = 0; b < si.ct; b++)
                ct[b] = (uint8_t)(c[b >> 3] >> (8 * (b & 7)));
        }
    };
    if (nthreads < 1)
        nthreads = 1;
    if ((size_t)nthreads > count / 64 + 1)
        nthreads = (int)(count / 64 + 1);
    if (nthreads == 1) {
        work(0, count);
        return CMD_OK;
    }
    std::vector<std::thread> th;
    const size_t per = (count + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; k++) {
        const size_t b = std::min(count, k * per), e = std::min(count, b + per);
        th.emplace_back(work, b, e);
    }
    for (auto &x : th)
        x.join();
    return CMD_OK;
}

}  // extern "C"
