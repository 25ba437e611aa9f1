// cmd_decrypt: drop-in for the reference's per-set CLI `decrypt_<set> [KATNUM]`
// (CPU/param/param6960119/src/decrypt.c:109-218).  With no path options it
// reads and writes the same relative paths the reference does:
//   ../../../kem/test_vectors/Cipher_Sk/{sk,ct}_<set>.bin   (util.c:13,30-58)
//   ../../results/output/errorstream0_<set>.bin           (decrypt.c:23)
// Exit status keeps the reference's codes: 0 success, -1 file error,
// -4 bad arguments (KATNUM <= 0 or unparsable).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cmd_b200.h"

static int usage(const char *argv0)
{
    fprintf(stderr,
            "Usage: %s <348864|460896|6688128|6960119|8192128> [KATNUM>0] [--sk PATH] [--ct PATH]\n"
            "          [--out PATH] [--path auto|plain|fused] [--device N] [--format text|binary]\n"
            "       %s --to-text BINARY_PATH TEXT_PATH   (binary errorstream -> text)\n",
            argv0, argv0);
    return CMD_E_ARG;
}

int main(int argc, char **argv)
{
    if (argc < 2)
        return usage(argv[0]);
    if (!strcmp(argv[1], "--to-text")) {
        if (argc != 4)
            return usage(argv[0]);
        const int rc = cmd_positions_to_errorstream(argv[2], argv[3]);
        if (rc != CMD_OK)
            fprintf(stderr, "convert: %s\n", cmd_last_error());
        return rc;
    }
    cmd_set set;
    if (cmd_set_from_name(argv[1], &set) != CMD_OK)
        return usage(argv[0]);
    long katnum = 5;  // the reference's default KATNUM (common.h)
    std::string dir = "../../../kem/test_vectors/Cipher_Sk/";
    std::string name = argv[1];
    if (!strncmp(name.c_str(), "mceliece", 8))
        name = name.substr(8);
    std::string sk = dir + "sk_" + name + ".bin", ct = dir + "ct_" + name + ".bin";
    std::string out = "../../results/output/errorstream0_" + name + ".bin";
    cmd_path path = CMD_PATH_AUTO;
    int device = 0;
    bool binary = false;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        auto val = [&]() -> const char * { return i + 1 < argc ? argv[++i] : nullptr; };
        if (a == "--format") {
            const char *v = val();
            if (!v || (strcmp(v, "text") && strcmp(v, "binary")))
                return usage(argv[0]);
            binary = !strcmp(v, "binary");
        } else if (a == "--sk" || a == "--ct" || a == "--out" || a == "--path" || a == "--device") {
            const char *v = val();
            if (!v)
                return usage(argv[0]);
            if (a == "--sk")
                sk = v;
            else if (a == "--ct")
                ct = v;
            else if (a == "--out")
                out = v;
            else if (a == "--device")
                device = atoi(v);
            else if (!strcmp(v, "plain"))
                path = CMD_PATH_PLAIN;
            else if (!strcmp(v, "fused"))
                path = CMD_PATH_FUSED;
            else if (!strcmp(v, "auto"))
                path = CMD_PATH_AUTO;
            else
                return usage(argv[0]);
        } else {
            char *end = nullptr;
            katnum = strtol(argv[i], &end, 10);
            if (argv[i][0] == '\0' || *end != '\0' || katnum <= 0)
                return usage(argv[0]);
        }
    }
    cmd_engine *eng = nullptr;
    int rc = cmd_engine_create(device, 0, &eng);
    if (rc != CMD_OK) {
        fprintf(stderr, "engine: %s\n", cmd_last_error());
        return rc;
    }
    double secs = 0;
    rc = binary ? cmd_decrypt_files_binary(eng, set, sk.c_str(), ct.c_str(), (size_t)katnum, out.c_str(), &secs)
                : cmd_decrypt_files(eng, set, sk.c_str(), ct.c_str(), (size_t)katnum, out.c_str(), path, &secs);
    if (rc != CMD_OK) {
        fprintf(stderr, "decrypt: %s\n", cmd_last_error());
    } else {
        printf("\n===== B200 batched decrypt =====\n");
        printf("ciphertexts processed : %ld\n", katnum);
        printf("device decrypt time   : %.6f s (host buffers, incl. transfers)\n", secs);
        printf("throughput            : %.2f cw/s\n", secs > 0 ? katnum / secs : 0.0);
        printf("errorstream           : %s%s\n", out.c_str(), binary ? " (binary positions)" : "");
    }
    cmd_engine_destroy(eng);
    return rc;
}
