/*
 * cmd_b200.h -- C ABI of the B200 (sm_100a) batched Classic McEliece
 * decryption engine.  A drop-in for the decrypt path of somesh-vas/CM_Decrypt_:
 * it reads the same sk_<set>.bin / ct_<set>.bin fixtures and produces the same
 * errorstream0_<set>.bin text, bit-exact with the reference CPU/ decoder,
 * decode failures included.
 *
 * The reference has no library API; its boundary is (i) the per-set CLI
 * `decrypt_<set> [KATNUM]` (CPU/param/param6960119/src/decrypt.c:109-218) with
 * fixed relative file paths, and (ii) the internal function trio synd/bm/root
 * over globals set up by initialisation()/compute_inverses()
 * (CPU/include/common/root.h:8-23, bm.h:14).  Each entry point below names the
 * reference interface it replaces.  Plain pointers and sizes only; status
 * codes, never exit().  Device pointers are marked d_*, host pointers h_*.
 * Streams are passed as void* (a cudaStream_t; NULL = the engine's stream).
 */
#ifndef CMD_B200_H
#define CMD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
/* 0 / -1 / -4 keep the reference's values (CPU/param/param6960119/include/
 * common.h:10-12: KAT_SUCCESS, KAT_FILE_OPEN_ERROR, KAT_CRYPTO_FAILURE). */
#define CMD_OK             0
#define CMD_E_FILE        -1  /* file missing, short, or unwritable          */
#define CMD_E_ARG         -4  /* bad argument (size, count, set, pointer)     */
#define CMD_E_CUDA        -5  /* a CUDA call failed; see cmd_last_error()     */
#define CMD_E_NOMEM       -6  /* host or device allocation failed             */
#define CMD_E_BUDGET      -7  /* refused: would exceed the engine HBM budget  */
#define CMD_E_BUSY        -8  /* serving queue full                           */
#define CMD_E_TIMEOUT     -9  /* a bounded wait gave up                       */
#define CMD_E_NODEVICE   -10  /* no CUDA device / kernels not loadable        */
#define CMD_E_KEYGEN     -11  /* key generation: attempt limit or self-check   */

/* ---- parameter sets (CPU/param/param<set>/include/common.h) ----------- */
typedef enum {
    CMD_348864 = 0,
    CMD_460896 = 1,
    CMD_6688128 = 2,
    CMD_6960119 = 3,
    CMD_8192128 = 4,
    CMD_NUM_SETS = 5
} cmd_set;

typedef struct {
    int32_t set_id;     /* 348864 ... 8192128                              */
    int32_t m;          /* GFBITS                                          */
    int32_t n;          /* SYS_N (support size = error-vector bits)        */
    int32_t t;          /* SYS_T                                           */
    int32_t ct_bytes;   /* crypto_kem_CIPHERTEXTBYTES (= SYND_BYTES)       */
    int32_t sk_bytes;   /* crypto_kem_SECRETKEYBYTES                       */
    int32_t sb;         /* 8*SYND_BYTES ciphertext bits used by synd()      */
    int32_t err_bytes;  /* n/8: bytes of one packed error vector           */
    int32_t err_words;  /* ceil(n/32): 32-bit words of one device error row */
} cmd_set_info;

/* Replaces the compile-time #defines of common.h with a runtime table. */
int cmd_set_info_get(cmd_set set, cmd_set_info *out);
/* "348864", "mceliece6960119", ... -> set.  CMD_E_ARG if unknown. */
int cmd_set_from_name(const char *name, cmd_set *out);

/* ---- engine ------------------------------------------------------------ */
typedef struct cmd_engine cmd_engine;
typedef struct cmd_key cmd_key;

/* One engine per GPU.  hbm_budget_bytes caps the device memory the engine
 * holds for keys and batch buffers (0 = 80% of free memory at creation). */
int cmd_engine_create(int device, size_t hbm_budget_bytes, cmd_engine **out);
void cmd_engine_destroy(cmd_engine *eng);
/* Bytes currently charged against the budget, and the budget itself. */
int cmd_engine_memory(const cmd_engine *eng, size_t *used, size_t *budget);
/* Text of the last error on this thread ("" if none). */
const char *cmd_last_error(void);
/* Kernel launches issued by this engine since creation (all streams). */
uint64_t cmd_engine_launch_count(const cmd_engine *eng);

/* ---- keys: secret-key expansion on the device ------------------------- */
/* Replaces initialisation() + support_gen() + compute_inverses()
 * (CPU/param/param6960119/src/util.c:60-100, CPU/src/common/root_13.c:181-211).
 * Parses sk (exactly sk_bytes), runs the Benes network, evaluates g on the
 * support and builds the device-resident tables: support L, 1/g(L_i)^2, the
 * syndrome table and the bitsliced support used by the root search.
 * CMD_E_BUDGET if the key does not fit the engine budget. */
int cmd_key_expand(cmd_engine *eng, cmd_set set, const uint8_t *h_sk,
                   size_t sk_len, cmd_key **out);
void cmd_key_free(cmd_key *key);
int cmd_key_set(const cmd_key *key, cmd_set *out);
size_t cmd_key_device_bytes(const cmd_key *key);
/* Parity hooks: copy the device-resident support L[n] (support_gen output),
 * Goppa g[t+1] and syndrome table [sb][2t] (inverse_elements) to the host. */
int cmd_key_support(const cmd_key *key, uint16_t *h_L, size_t n);
int cmd_key_goppa(const cmd_key *key, uint16_t *h_g, size_t t_plus_1);
int cmd_key_synd_table(const cmd_key *key, uint16_t *h_tab, size_t entries);

/* ---- batched decrypt --------------------------------------------------- */
/* Path selector: CMD_PATH_PLAIN runs the three per-stage kernels (syndrome,
 * Berlekamp-Massey, root search + pack); CMD_PATH_FUSED runs the fused
 * bitsliced kernel; CMD_PATH_TILE runs the serving loop's latency kernels
 * (syndromes by the transposed additive FFT, a CTA per 32-ciphertext tile
 * for Berlekamp-Massey, a warp per ciphertext for the root search);
 * CMD_PATH_AUTO lets the engine's tuner choose.  Graph capture takes AUTO,
 * PLAIN and FUSED. */
typedef enum { CMD_PATH_AUTO = 0, CMD_PATH_PLAIN = 1, CMD_PATH_FUSED = 2, CMD_PATH_TILE = 3 } cmd_path;

/* Replaces the per-ciphertext loop memcpy -> synd -> bm -> root ->
 * build_error_vector (CPU/param/param6960119/src/decrypt.c:163-177, 43-53).
 * h_cts: count * ct_bytes, raw concatenation (the ct_<set>.bin layout).
 * h_err: count * err_bytes; bit i of vector c is set iff position i is flagged
 * (the reference's error_vector layout).  h_weight (may be NULL): flagged
 * positions per ciphertext.  Synchronous; host buffers may be pageable.
 * When h_err is pinned memory the GPU maps (cudaHostAlloc / cudaMallocHost,
 * or registered with a device mapping; 2-byte aligned, all count * err_bytes
 * in one allocation), batches of 65,536 ciphertexts or more have the kernels
 * store the rows into it directly while they run, with no copy after them. */
int cmd_decrypt_batch(cmd_engine *eng, const cmd_key *key, cmd_path path,
                      const uint8_t *h_cts, size_t count, uint8_t *h_err,
                      uint16_t *h_weight);

/* Device-resident form: d_cts as above; d_err is count rows of err_words
 * 32-bit words (little-endian, so the first err_bytes bytes of a row equal the
 * host layout; bits >= n are zero).  Asynchronous on `stream`. */
int cmd_decrypt_device(cmd_engine *eng, const cmd_key *key, cmd_path path,
                       const uint8_t *d_cts, size_t count, uint32_t *d_err,
                       uint16_t *d_weight, void *stream);

/* Mixed batch in one launch: ciphertext c belongs to keys[h_key_idx[c]]; its
 * bytes start at d_cts + h_ct_off[c] and its error row at
 * d_err + h_err_off[c] (in 32-bit words).  Keys may be of different sets.
 * Always runs the fused kernel.  Asynchronous on `stream`. */
int cmd_decrypt_mixed_device(cmd_engine *eng, const cmd_key *const *keys,
                             size_t nkeys, const uint32_t *h_key_idx,
                             const uint8_t *d_cts, const uint64_t *h_ct_off,
                             size_t count, uint32_t *d_err,
                             const uint64_t *h_err_off, uint16_t *d_weight,
                             void *stream);

/* Allocation-free decrypt.  No counterpart in the reference: it exists for
 * callers that must not have the library allocate device memory -- hosts whose
 * device memory belongs to another allocator (e.g. a framework's pool), or
 * latency-critical loops that cannot afford a cudaMalloc/cudaFree and the
 * synchronisation it brings.  It runs the plain three-kernel path (same
 * results as cmd_decrypt_device with CMD_PATH_PLAIN) but keeps the syndrome
 * and locator intermediates in a fixed device array inside the library,
 * sized for CMD_NOALLOC_MAX_CTS ciphertexts per call (about 3 MiB, held by
 * every GPU that loads the library until the process exits).  The caller
 * passes the expanded key, device ciphertexts (count * ct_bytes) and device
 * outputs (count rows of err_words words; weights may be NULL).  count above
 * the maximum returns CMD_E_ARG.  cmd_engine_create looks up the array's
 * device address and loads the array and the plain kernels onto the device,
 * so the call itself loads and allocates nothing.  Calls share the array:
 * calls that overlap on the GPU (concurrent streams or threads) race, so
 * serialise them.  The caller's current device is left as it was.
 * Asynchronous on `stream` (NULL = the key's engine stream). */
#define CMD_NOALLOC_MAX_CTS 4096
int cmd_decrypt_plain_noalloc(const cmd_key *key, const uint8_t *d_cts,
                              size_t count, uint32_t *d_err,
                              uint16_t *d_weight, void *stream);

/* ---- per-stage parity hooks (device buffers, asynchronous) ------------- */
/* synd(): d_synd = count rows of 2t u16 (CPU/param/param6960119/src/
 * util.c:102-114). */
int cmd_stage_synd(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts,
                   size_t count, uint16_t *d_synd, void *stream);
/* synd() by the serving path's method (the transposed additive FFT over the
 * key's support network, no syndrome table): the same count rows of 2t u16
 * (CPU/param/param6960119/src/util.c:102-114). */
int cmd_stage_synd_fft(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts,
                       size_t count, uint16_t *d_synd, void *stream);
/* bm(): d_loc = count rows of t+1 u16, reversed as bm() writes them
 * (CPU/src/common/bm.c:12-68). */
int cmd_stage_bm(cmd_engine *eng, cmd_set set, const uint16_t *d_synd,
                 size_t count, uint16_t *d_loc, void *stream);
/* root() + build_error_vector: flagged-position rows (err_words words) and
 * weights from locators (CPU/src/common/root_13.c:233-240, decrypt.c:43-53). */
int cmd_stage_root(cmd_engine *eng, const cmd_key *key, const uint16_t *d_loc,
                   size_t count, uint32_t *d_err, uint16_t *d_weight,
                   void *stream);
/* root() images themselves: count rows of n u16 (for stage-level diffs). */
int cmd_stage_root_images(cmd_engine *eng, const cmd_key *key,
                          const uint16_t *d_loc, size_t count,
                          uint16_t *d_images, void *stream);

/* ---- errorstream (text) ------------------------------------------------ */
/* write_error_positions (CPU/param/param6960119/src/decrypt.c:55-66): one
 * line per vector, " %d" per flagged position ascending, then '\n'.
 * Returns CMD_OK and the byte count in *out_len; CMD_E_ARG if cap is short
 * (with *out_len = bytes needed). */
int cmd_errorstream_format(cmd_set set, const uint8_t *h_err, size_t count,
                           char *out, size_t cap, size_t *out_len);
/* Writes (append != 0: appends) the text to path.  CMD_E_FILE on failure. */
int cmd_errorstream_write(cmd_set set, const uint8_t *h_err, size_t count,
                          const char *path, int append);

/* ---- error positions and the binary errorstream (no reference counterpart) */
/* The decrypt result as error positions: row c of the output holds t+1 u16,
 * the weight w, then the w flagged positions in ascending order (the numbers
 * write_error_positions prints for that ciphertext), then 0xFFFF.  The
 * weight never exceeds t (the reversed locator has degree exactly t).  Runs
 * the fused kernel, which writes the rows directly: 2(t+1) bytes per
 * ciphertext instead of n/8 (240 vs 870 bytes for 6960119).
 * cmd_decrypt_positions takes host buffers (like cmd_decrypt_batch),
 * cmd_decrypt_positions_device device buffers, asynchronous on `stream`. */
int cmd_decrypt_positions(cmd_engine *eng, const cmd_key *key, const uint8_t *h_cts,
                          size_t count, uint16_t *h_pos);
int cmd_decrypt_positions_device(cmd_engine *eng, const cmd_key *key,
                                 const uint8_t *d_cts, size_t count, uint16_t *d_pos,
                                 void *stream);
/* The errorstream text of positions rows: the same bytes cmd_errorstream_format
 * gives for the equivalent error vectors. */
int cmd_positions_format(cmd_set set, const uint16_t *h_pos, size_t count,
                         char *out, size_t cap, size_t *out_len);
/* Binary errorstream: a 24-byte header -- "CMDPOS01", the set id (u32 LE,
 * e.g. 6960119), t (u32 LE), the row count (u64 LE) -- then the positions
 * rows (t+1 u16 LE each).  Writing it is a copy of the rows; append != 0 adds
 * rows to an existing file of the same set.  CMD_E_FILE on I/O errors or a
 * foreign file. */
int cmd_positions_write(cmd_set set, const uint16_t *h_pos, size_t count,
                        const char *path, int append);
/* Converts a binary errorstream into the reference's errorstream text. */
int cmd_positions_to_errorstream(const char *binary_path, const char *text_path);

/* ---- KEM decapsulation (no counterpart in the reference) --------------- */
/* The reference encapsulates only (kem/common/core/operations.c:15-34:
 * C = [I | T] e, K = SHAKE256(1 || e || C), 32 bytes).  Decapsulation with
 * implicit rejection: e = the decrypt of C (as cmd_decrypt_*); accept iff the
 * padding bits of C above mt are zero, wt(e) == t and C == [I | T] e; then
 * K = SHAKE256(b || v || C) with b = accept and v = e, or v = the secret
 * key's n/8-byte string s when rejected.  The re-encoding check reads every
 * column of T for every ciphertext, and v is selected with masks, so the
 * work does not depend on e.  The first call for a key derives T on the
 * device from the key's support and Goppa polynomial (the key generation's
 * elimination) and keeps it there, charged to the engine's budget (1.1 MB for
 * 6960119); cmd_key_prepare_decap does that step ahead of time.  CMD_E_ARG
 * when the key's parity-check matrix has no systematic form.
 * keys: 32 bytes per ciphertext; accept (may be NULL): 1 byte each. */
int cmd_key_prepare_decap(cmd_engine *eng, cmd_key *key);
int cmd_kem_decap(cmd_engine *eng, cmd_key *key, const uint8_t *h_cts, size_t count,
                  uint8_t *h_keys, uint8_t *h_accept);
int cmd_kem_decap_device(cmd_engine *eng, cmd_key *key, const uint8_t *d_cts, size_t count,
                         uint8_t *d_keys, uint8_t *d_accept, void *stream);

/* ---- file contract ----------------------------------------------------- */
/* Replaces `decrypt_<set> KATNUM` (decrypt.c:109-218): reads one sk
 * (sk_bytes) and katnum ciphertexts from the given files, decrypts on the GPU
 * and writes the errorstream.  CMD_E_FILE (-1) if a file is missing or short,
 * CMD_E_ARG (-4) for katnum == 0.  *out_seconds (may be NULL) receives the
 * device decrypt time. */
int cmd_decrypt_files(cmd_engine *eng, cmd_set set, const char *sk_path,
                      const char *ct_path, size_t katnum,
                      const char *errorstream_path, cmd_path path,
                      double *out_seconds);
/* As cmd_decrypt_files, writing the binary errorstream (positions rows, see
 * cmd_positions_write) instead of the text; cmd_positions_to_errorstream
 * turns it into the reference's text. */
int cmd_decrypt_files_binary(cmd_engine *eng, cmd_set set, const char *sk_path,
                             const char *ct_path, size_t katnum,
                             const char *positions_path, double *out_seconds);

/* ---- serving loop (no reference counterpart) ---------------------------- */
/* Continuous batching of single-ciphertext decapsulation requests over many
 * keys and parameter sets.  A dispatcher forms a batch whenever one of
 * `slots` batch slots is free and requests wait: at once when nothing is on
 * the GPU, otherwise after the oldest request has waited max_wait_us for
 * batch-mates (or the batch is full).  Batches of different slots overlap on
 * the device.  Keys registered with cmd_server_add_key are expanded on first
 * use and stay resident; least recently used keys are evicted when the
 * engine's HBM budget is full; when one batch needs more keys than fit at
 * once, the requests of the keys that did not fit wait for the next batch.
 * Batches of at least fused_threshold requests run the fused kernel, smaller
 * ones the latency kernels (one short pass per ciphertext; fused_threshold 0:
 * always the latency kernels).  Each slot has its own stream: give the process
 * at least as many hardware work queues (CUDA_DEVICE_MAX_CONNECTIONS, read at
 * context creation, default 8) as slots plus the streams of other work, or
 * batches queue behind each other on the device. */
typedef struct cmd_server cmd_server;
typedef struct {
    uint32_t max_batch;          /* requests per batch, 1..65536              */
    uint32_t slots;              /* batches in flight, 1..16                  */
    uint32_t max_wait_us;        /* batching delay bound while the GPU is busy */
    uint32_t queue_capacity;     /* waiting requests before CMD_E_BUSY        */
    uint32_t fused_threshold;    /* batch size from which the fused kernel runs */
    uint32_t record_completions; /* 1: queue a cmd_completion per request     */
} cmd_server_config;
typedef struct {
    uint64_t tag;        /* caller's tag from cmd_server_submit           */
    int32_t status;      /* CMD_OK or the batch's error                   */
    uint16_t weight;     /* flagged positions                             */
    uint16_t reserved;
    uint64_t latency_ns; /* arrival -> result in the caller's buffer       */
} cmd_completion;
typedef struct {
    uint64_t submitted, completed, refused, batches, fused_batches, resident_keys;
    double mean_batch, p50_us, p99_us, max_us, mean_us;
    double decaps_per_s;  /* completed / (last completion - first arrival)  */
    double offered_per_s; /* cmd_server_loadgen: arrival rate actually offered */
    double gpu_p50_us, gpu_p99_us; /* per batch: device time from the input copy
                                      to the end of the result copy          */
    double wait_p50_us, wait_p99_us; /* per request: arrival -> batch launch  */
    double dispatch_busy;  /* host time forming and launching batches / interval */
    double complete_busy;  /* host time delivering results / interval          */
    double mean_inflight;  /* batches on the GPU when a batch is launched (incl.) */
} cmd_server_stats;

int cmd_server_create(cmd_engine *eng, const cmd_server_config *cfg, cmd_server **out);
/* Finishes every accepted request, then releases the server and its keys. */
void cmd_server_destroy(cmd_server *srv);
int cmd_server_add_key(cmd_server *srv, cmd_set set, const uint8_t *h_sk, size_t sk_len,
                       uint32_t *key_id);
/* Registers [h_rows, h_rows + bytes) for result rows.  A request queued
 * afterwards whose result buffer (err_bytes from an even address) lies in a
 * registered range has its row stored there by the GPU itself on the latency
 * kernels' path: the row crosses PCIe while the batch runs, and nothing is
 * copied on the host when it completes.  Memory the GPU already maps (pinned
 * by cudaHostAlloc / cudaMallocHost, or registered as mapped) is used as it
 * is; other memory is pinned and mapped here (cudaHostRegister) and
 * unregistered by cmd_server_destroy.  The range must stay allocated until
 * cmd_server_destroy returns.  Other requests, and fused-kernel batches,
 * take the staged copy. */
int cmd_server_register_rows(cmd_server *srv, uint8_t *h_rows, size_t bytes);
/* Queues one ciphertext (ct_bytes of key_id's set); on completion err_bytes
 * of packed error bits are written to h_err_out (may be NULL).  Non-blocking;
 * CMD_E_BUSY when queue_capacity requests are waiting. */
int cmd_server_submit(cmd_server *srv, uint32_t key_id, const uint8_t *h_ct, uint8_t *h_err_out,
                      uint64_t tag);
/* Queues n requests under one lock, in order: request i is key_ids[i], the
 * ciphertext at h_cts + i * ct_stride, its result (when h_err_base is not
 * NULL) at h_err_base + i * err_stride, tag tags[i] (i when tags is NULL).
 * *accepted = how many were queued before the queue filled; CMD_E_BUSY when
 * that is fewer than n (the rest are refused and counted as such). */
int cmd_server_submit_many(cmd_server *srv, size_t n, const uint32_t *key_ids, const uint8_t *h_cts,
                           size_t ct_stride, uint8_t *h_err_base, size_t err_stride, const uint64_t *tags,
                           size_t *accepted);
/* Up to max completions (waits up to timeout_us for the first).  Returns the
 * server's sticky status (CMD_OK unless a batch failed). */
int cmd_server_poll(cmd_server *srv, cmd_completion *out, size_t max, size_t *n, uint32_t timeout_us);
/* Waits until every accepted request has completed (CMD_E_TIMEOUT after timeout_ms). */
int cmd_server_drain(cmd_server *srv, uint32_t timeout_ms);
int cmd_server_stats_get(cmd_server *srv, cmd_server_stats *out, int reset);
/* Open-loop Poisson load for `seconds` at rate_per_s: request i uses
 * key_ids[i % pool] and ciphertext i % pool (ct_stride bytes apart) and writes
 * its result to err_pool row i % pool (err_stride bytes apart; may be NULL).
 * Each request is queued with its scheduled arrival time, so its latency
 * counts from when it was due; the generator queues all requests due at
 * once.  Statistics are reset first and returned in *out after a full drain. */
int cmd_server_loadgen(cmd_server *srv, const uint32_t *key_ids, const uint8_t *cts, size_t ct_stride,
                       uint8_t *err_pool, size_t err_stride, size_t pool, double rate_per_s,
                       double seconds, uint64_t seed, cmd_server_stats *out);

/* ---- key generation (kem/common/core/operations.c:36-107) -------------- */
/* crypto_kem_keypair with randombytes() yielding the caller's 32-byte seed:
 * pk receives mt rows of (n - mt + 7)/8 bytes (pk_gen.c:145-146), sk the
 * reference's secret-key layout (seed | pivots | g | control bits | s).  A
 * rejected attempt continues with the next seed of the expansion, as the
 * reference's loop does, so a seed yields the reference's key pair; the
 * secret key's first 32 bytes are the seed of the accepted attempt.
 * *attempts (may be NULL) receives the attempts taken.  Every stage runs on
 * the GPU; field arithmetic is table-free, the elimination and the control
 * bits are not constant-time (see keygen.cu).
 * CMD_E_KEYGEN if the attempt limit is reached or the control bits fail their
 * self-check. */
int cmd_kem_keypair(cmd_engine *eng, cmd_set set, const uint8_t *h_seed, uint8_t *h_pk,
                    uint8_t *h_sk, uint32_t *attempts);
/* count (1..4096) seeds of 32 bytes: key pairs in pk/sk rows of the sizes
 * above; attempts[i] per key (may be NULL).  Up to four consecutive attempts
 * of a key run side by side and the first accepted one is kept, so results
 * and attempt counts are those of the sequential loop.  A key is given up
 * (CMD_E_KEYGEN) once at least max_attempts (0 = 1000) have failed. */
int cmd_kem_keypair_batch(cmd_engine *eng, cmd_set set, const uint8_t *h_seeds, size_t count,
                          uint8_t *h_pk, uint8_t *h_sk, uint32_t *attempts, uint32_t max_attempts);

/* ---- fused-kernel tuning and graph replay (no reference counterpart) --- */
/* Picks the fused kernel's launch configuration for key's set on this GPU
 * (warps per CTA 4|8, equal-share or full rounds) by timing the candidates on
 * sample_count ciphertexts (0 = about three waves; pass the batch size the
 * caller runs: the winner depends on how that size fills whole rounds of the
 * resident warps, and each size is cached apart), then the batch size below
 * which CMD_PATH_AUTO takes the tile kernels instead (five warps per
 * 32-ciphertext tile for Berlekamp-Massey rather than the fused kernel's
 * one), from timings of both at 256 .. 65,536 ciphertexts.  Results are
 * cached in the engine and in $CMD_TUNE_CACHE (JSON keyed by GPU name and
 * set); a cached entry is reused unless force != 0. */
int cmd_tune(cmd_engine *eng, const cmd_key *key, size_t sample_count, int force);
int cmd_engine_fused_config(cmd_engine *eng, cmd_set set, int *wpb, int *balanced,
                            double *ns_per_ct);
/* The tuned batch size below which CMD_PATH_AUTO runs the tile kernels (0:
 * never). */
int cmd_engine_tile_below(cmd_engine *eng, cmd_set set, uint32_t *tile_below);
int cmd_engine_set_fused_config(cmd_engine *eng, cmd_set set, int wpb, int balanced);

/* A decrypt over fixed device buffers captured as a CUDA graph and replayed
 * with cmd_graph_launch (asynchronous on `stream`, NULL = engine stream).
 * A fused-path graph owns its work counter; a plain-path graph uses the
 * engine's scratch, so do not replay it concurrently with other plain-path
 * work of the same engine. */
typedef struct cmd_graph cmd_graph;
int cmd_graph_capture(cmd_engine *eng, const cmd_key *key, cmd_path path,
                      const uint8_t *d_cts, size_t count, uint32_t *d_err,
                      uint16_t *d_weight, cmd_graph **out);
int cmd_graph_launch(cmd_graph *graph, void *stream);
void cmd_graph_destroy(cmd_graph *graph);

/* ---- measurement (no reference counterpart) ---------------------------- */
/* Integer-ALU roofline denominator: the device's sustained lop3.b32 rate in
 * lane-operations per second (32 per warp instruction), measured with
 * independent dependency chains on every SM. */
int cmd_bench_int_peak(cmd_engine *eng, double *lop3_lane_ops_per_s);

/* ---- synthetic workloads (no reference counterpart: fixture tooling) --- */
/* Derives a secret key for `set` from a 64-bit seed: the Goppa polynomial of
 * the base key h_base_sk translated by a seed-chosen field element (which
 * keeps it irreducible) and fresh seed-drawn Benes control bits, retried
 * until the first mt support columns form an invertible block.  h_sk_out
 * receives sk_bytes.  h_base_sk may be NULL for set 0..4 built-in bases. */
int cmd_synth_key(cmd_set set, const uint8_t *h_base_sk, uint64_t seed,
                  uint8_t *h_sk_out);
/* Public data for encryption: the systematic parity-check matrix built from
 * sk; opaque handle. */
typedef struct cmd_pubkey cmd_pubkey;
int cmd_synth_pubkey(cmd_set set, const uint8_t *h_sk, cmd_pubkey **out);
void cmd_synth_pubkey_free(cmd_pubkey *pk);
/* The T block of the systematic public key [I | T]: column i (i < n - mt)
 * in words_per_col u64 (bit r = row r, r < mt) at out + i * words_per_col.
 * out == NULL only reports words_per_col. */
int cmd_pubkey_columns(const cmd_pubkey *pk, uint64_t *out, size_t cap_words,
                       size_t *words_per_col);
/* count ciphertexts: ciphertext i is valid (an error vector of weight exactly
 * t, positions uniform over [0,n), seeded by (seed, i)) unless
 * i is drawn malformed with probability malformed_permille/1000, in which case
 * it is a uniform random mt-bit string (padding bits zero).  h_err_out (may be
 * NULL) gets the planted error vectors (all-zero rows for malformed ones),
 * h_valid_out (may be NULL) 1/0 per ciphertext. */
int cmd_synth_ciphertexts(const cmd_pubkey *pk, uint64_t seed, size_t count,
                          uint32_t malformed_permille, uint8_t *h_cts_out,
                          uint8_t *h_err_out, uint8_t *h_valid_out,
                          int nthreads);

#ifdef __cplusplus
}
#endif
#endif /* CMD_B200_H */
