// Errorstream text and the file contract of the reference decoder.
//
// Text format (write_error_positions, CPU/param/param6960119/src/decrypt.c:
// 55-66): per ciphertext, " %d" for every flagged position in ascending
// order, then '\n'.  Files: sk_<set>.bin holds one secret key, ct_<set>.bin
// katnum raw ciphertexts (util.c:30-58 reads exactly those sizes).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"

namespace {

// Appends " <pos>" for every set bit of an n-bit little-endian vector.
size_t format_row(const uint8_t *e, int n, char *out)
{
    char *p = out;
    for (int w = 0; w < n / 8; w += 8) {
        uint64_t x = 0;
        const int nb = std::min(8, n / 8 - w);
        memcpy(&x, e + w, nb);
        while (x) {
            const int pos = 8 * w + __builtin_ctzll(x);
            x &= x - 1;
            char buf[8];
            int len = 0, v = pos;
            do {
                buf[len++] = (char)('0' + v % 10);
                v /= 10;
            } while (v);
            *p++ = ' ';
            while (len)
                *p++ = buf[--len];
        }
    }
    *p++ = '\n';
    return (size_t)(p - out);
}

size_t row_bound(int n) { return 1 + 6 * (size_t)n; }

// " %d" per position, then '\n' (the text of format_row, from a positions row).
size_t format_positions(const uint16_t *row, int t, char *out)
{
    char *p = out;
    const int w = row[0] < t ? row[0] : t;
    for (int i = 0; i < w; i++) {
        char buf[8];
        int len = 0, v = row[1 + i];
        do {
            buf[len++] = (char)('0' + v % 10);
            v /= 10;
        } while (v);
        *p++ = ' ';
        while (len)
            *p++ = buf[--len];
    }
    *p++ = '\n';
    return (size_t)(p - out);
}

constexpr char POS_MAGIC[8] = {'C', 'M', 'D', 'P', 'O', 'S', '0', '1'};

struct PosHeader {
    char magic[8];
    uint32_t set_id;  // e.g. 6960119
    uint32_t t;       // row = t+1 u16
    uint64_t rows;
};
static_assert(sizeof(PosHeader) == 24, "positions header layout");

}  // namespace

extern "C" {

int cmd_errorstream_format(cmd_set set, const uint8_t *h_err, size_t count, char *out, size_t cap, size_t *out_len)
{
    if (set < 0 || set >= cmd::NSETS || (count && !h_err) || !out_len)
        return CMD_E_ARG;
    const cmd::SetInfo si = cmd::set_info(set);
    std::vector<char> row(row_bound(si.n));
    size_t pos = 0;
    bool fits = true;
    for (size_t c = 0; c < count; c++) {
        const size_t len = format_row(h_err + c * (si.n / 8), si.n, row.data());
        if (fits && out && pos + len <= cap)
            memcpy(out + pos, row.data(), len);
        else
            fits = false;
        pos += len;
    }
    *out_len = pos;
    return fits ? CMD_OK : CMD_E_ARG;
}

int cmd_errorstream_write(cmd_set set, const uint8_t *h_err, size_t count, const char *path, int append)
{
    if (set < 0 || set >= cmd::NSETS || (count && !h_err) || !path)
        return CMD_E_ARG;
    const cmd::SetInfo si = cmd::set_info(set);
    FILE *f = fopen(path, append ? "ab" : "wb");
    if (!f) {
        cmd::set_last_error(std::string("cannot open errorstream ") + path);
        return CMD_E_FILE;
    }
    std::vector<char> buf;
    buf.reserve(1 << 20);
    std::vector<char> row(row_bound(si.n));
    int rc = CMD_OK;
    for (size_t c = 0; c < count && rc == CMD_OK; c++) {
        const size_t len = format_row(h_err + c * (si.n / 8), si.n, row.data());
        buf.insert(buf.end(), row.data(), row.data() + len);
        if (buf.size() >= (1 << 20) || c + 1 == count) {
            if (fwrite(buf.data(), 1, buf.size(), f) != buf.size())
                rc = CMD_E_FILE;
            buf.clear();
        }
    }
    if (fclose(f) != 0)
        rc = CMD_E_FILE;
    return rc;
}

int cmd_positions_format(cmd_set set, const uint16_t *h_pos, size_t count, char *out, size_t cap, size_t *out_len)
{
    if (set < 0 || set >= cmd::NSETS || (count && !h_pos) || !out_len)
        return CMD_E_ARG;
    const cmd::SetInfo si = cmd::set_info(set);
    std::vector<char> row(row_bound(si.t));
    size_t pos = 0;
    bool fits = true;
    for (size_t c = 0; c < count; c++) {
        const size_t len = format_positions(h_pos + c * (si.t + 1), si.t, row.data());
        if (fits && out && pos + len <= cap)
            memcpy(out + pos, row.data(), len);
        else
            fits = false;
        pos += len;
    }
    *out_len = pos;
    return fits ? CMD_OK : CMD_E_ARG;
}

int cmd_positions_write(cmd_set set, const uint16_t *h_pos, size_t count, const char *path, int append)
{
    if (set < 0 || set >= cmd::NSETS || (count && !h_pos) || !path)
        return CMD_E_ARG;
    const cmd::SetInfo si = cmd::set_info(set);
    PosHeader h;
    memcpy(h.magic, POS_MAGIC, 8);
    h.set_id = (uint32_t)si.id;
    h.t = (uint32_t)si.t;
    h.rows = 0;
    FILE *f = nullptr;
    if (append) {
        f = fopen(path, "r+b");
        if (f) {
            PosHeader old;
            if (fread(&old, sizeof old, 1, f) != 1 || memcmp(old.magic, POS_MAGIC, 8) || old.set_id != h.set_id ||
                old.t != h.t) {
                fclose(f);
                cmd::set_last_error(std::string("not a positions file of this set: ") + path);
                return CMD_E_FILE;
            }
            h.rows = old.rows;
        }
    }
    if (!f)
        f = fopen(path, "w+b");
    if (!f) {
        cmd::set_last_error(std::string("cannot open ") + path);
        return CMD_E_FILE;
    }
    const size_t row = (size_t)si.t + 1;
    bool ok = fseek(f, (long)(sizeof h + h.rows * row * 2), SEEK_SET) == 0 &&
              fwrite(h_pos, row * 2, count, f) == count;
    h.rows += count;
    ok = ok && fseek(f, 0, SEEK_SET) == 0 && fwrite(&h, sizeof h, 1, f) == 1;
    if (fclose(f) != 0)
        ok = false;
    return ok ? CMD_OK : CMD_E_FILE;
}

int cmd_positions_to_errorstream(const char *binary_path, const char *text_path)
{
    if (!binary_path || !text_path)
        return CMD_E_ARG;
    FILE *f = fopen(binary_path, "rb");
    if (!f) {
        cmd::set_last_error(std::string("cannot open ") + binary_path);
        return CMD_E_FILE;
    }
    PosHeader h;
    cmd_set set = (cmd_set)-1;
    if (fread(&h, sizeof h, 1, f) == 1 && !memcmp(h.magic, POS_MAGIC, 8)) {
        for (int s = 0; s < cmd::NSETS; s++)
            if ((uint32_t)cmd::set_info(s).id == h.set_id && (uint32_t)cmd::set_info(s).t == h.t)
                set = (cmd_set)s;
    }
    if (set < 0) {
        fclose(f);
        cmd::set_last_error(std::string("not a positions file: ") + binary_path);
        return CMD_E_FILE;
    }
    FILE *o = fopen(text_path, "wb");
    if (!o) {
        fclose(f);
        cmd::set_last_error(std::string("cannot open ") + text_path);
        return CMD_E_FILE;
    }
    const size_t row = (size_t)h.t + 1;
    const size_t batch = 4096;
    std::vector<uint16_t> in(batch * row);
    std::vector<char> text;
    int rc = CMD_OK;
    for (uint64_t done = 0; done < h.rows && rc == CMD_OK;) {
        const size_t n = (size_t)std::min<uint64_t>(batch, h.rows - done);
        if (fread(in.data(), row * 2, n, f) != n) {
            cmd::set_last_error(std::string("short positions file: ") + binary_path);
            rc = CMD_E_FILE;
            break;
        }
        size_t len = 0;
        cmd_positions_format(set, in.data(), n, nullptr, 0, &len);
        text.resize(len);
        cmd_positions_format(set, in.data(), n, text.data(), len, &len);
        if (fwrite(text.data(), 1, len, o) != len)
            rc = CMD_E_FILE;
        done += n;
    }
    fclose(f);
    if (fclose(o) != 0)
        rc = CMD_E_FILE;
    return rc;
}

int cmd_decrypt_files(cmd_engine *eng, cmd_set set, const char *sk_path, const char *ct_path, size_t katnum,
                      const char *errorstream_path, cmd_path path, double *out_seconds)
{
    if (!eng || set < 0 || set >= cmd::NSETS || !sk_path || !ct_path || !errorstream_path)
        return CMD_E_ARG;
    if (katnum == 0)
        return CMD_E_ARG;  // the reference rejects KATNUM <= 0 with KAT_CRYPTO_FAILURE
    const cmd::SetInfo si = cmd::set_info(set);
    std::vector<uint8_t> sk(si.sk), cts(katnum * si.ct);
    FILE *fs = fopen(sk_path, "rb");
    FILE *fc = fopen(ct_path, "rb");
    const bool ok = fs && fc && fread(sk.data(), si.sk, 1, fs) == 1 && fread(cts.data(), si.ct, katnum, fc) == katnum;
    if (fs)
        fclose(fs);
    if (fc)
        fclose(fc);
    if (!ok) {
        cmd::set_last_error(std::string("cannot read ") + sk_path + " / " + ct_path);
        return CMD_E_FILE;
    }
    cmd_key *key = nullptr;
    int rc = cmd_key_expand(eng, set, sk.data(), sk.size(), &key);
    if (rc)
        return rc;
    std::vector<uint8_t> err(katnum * (si.n / 8));
    const auto t0 = std::chrono::steady_clock::now();
    rc = cmd_decrypt_batch(eng, key, path, cts.data(), katnum, err.data(), nullptr);
    const auto t1 = std::chrono::steady_clock::now();
    cmd_key_free(key);
    if (out_seconds)
        *out_seconds = std::chrono::duration<double>(t1 - t0).count();
    if (rc)
        return rc;
    return cmd_errorstream_write(set, err.data(), katnum, errorstream_path, 0);
}

}  // extern "C"

extern "C" int cmd_decrypt_files_binary(cmd_engine *eng, cmd_set set, const char *sk_path, const char *ct_path,
                                        size_t katnum, const char *positions_path, double *out_seconds)
{
    if (!eng || set < 0 || set >= cmd::NSETS || !sk_path || !ct_path || !positions_path)
        return CMD_E_ARG;
    if (katnum == 0)
        return CMD_E_ARG;
    const cmd::SetInfo si = cmd::set_info(set);
    std::vector<uint8_t> sk(si.sk), cts(katnum * si.ct);
    FILE *fs = fopen(sk_path, "rb");
    FILE *fc = fopen(ct_path, "rb");
    const bool ok = fs && fc && fread(sk.data(), si.sk, 1, fs) == 1 && fread(cts.data(), si.ct, katnum, fc) == katnum;
    if (fs)
        fclose(fs);
    if (fc)
        fclose(fc);
    if (!ok) {
        cmd::set_last_error(std::string("cannot read ") + sk_path + " / " + ct_path);
        return CMD_E_FILE;
    }
    cmd_key *key = nullptr;
    int rc = cmd_key_expand(eng, set, sk.data(), sk.size(), &key);
    if (rc)
        return rc;
    std::vector<uint16_t> pos(katnum * (si.t + 1));
    const auto t0 = std::chrono::steady_clock::now();
    rc = cmd_decrypt_positions(eng, key, cts.data(), katnum, pos.data());
    const auto t1 = std::chrono::steady_clock::now();
    cmd_key_free(key);
    if (out_seconds)
        *out_seconds = std::chrono::duration<double>(t1 - t0).count();
    if (rc)
        return rc;
    return cmd_positions_write(set, pos.data(), katnum, positions_path, 0);
}
