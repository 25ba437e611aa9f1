// Autotuner for the fused kernel and CUDA-graph capture/replay of a decrypt.
//
// Tuner: for one parameter set on one GPU it times the candidate launch
// configurations (warps per CTA x round schedule) on a device batch and keeps
// the fastest; then it times the fastest against the tile kernels (five warps
// per 32-ciphertext tile for Berlekamp-Massey instead of one) at growing batch
// sizes and records the size from which the fused kernel wins, below which
// CMD_PATH_AUTO takes the tile kernels.  The decrypt kernels' instruction stream does not depend on
// the ciphertext contents, so the sample is a constant byte pattern.  Choices
// are cached per engine and persisted as JSON keyed by (GPU name, set) in
// $CMD_TUNE_CACHE (default ~/.cache/cmd_b200/tune.json).
//
// Graphs: a decrypt over fixed device buffers is captured once and replayed,
// which removes the per-call host work (argument checks, round sizing,
// occupancy lookups) from a launch-bound loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <sys/stat.h>

#include "engine.h"

namespace cmd {

size_t plain_scratch_bytes(int set, size_t count);
cudaError_t fused_prepare(cmd_engine *eng, int set);

static std::string cache_path()
{
    if (const char *p = getenv("CMD_TUNE_CACHE"))
        return p;
    const char *home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/cmd_b200/tune.json";
}

// Minimal reader/writer for
// {"key": {"wpb": n, "balanced": b, "ns_per_ct": x, "tile_below": c}, ...};
// an entry without tile_below (an older tuner's) is tuned again.
static std::map<std::string, FusedConfig> load_cache()
{
    std::map<std::string, FusedConfig> out;
    FILE *f = fopen(cache_path().c_str(), "rb");
    if (!f)
        return out;
    std::string s;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0)
        s.append(buf, n);
    fclose(f);
    size_t pos = 0;
    while ((pos = s.find('"', pos)) != std::string::npos) {
        const size_t end = s.find('"', pos + 1);
        if (end == std::string::npos)
            break;
        const std::string key = s.substr(pos + 1, end - pos - 1);
        const size_t ob = s.find('{', end), cb = s.find('}', end);
        if (ob == std::string::npos || cb == std::string::npos || ob > cb) {
            pos = end + 1;
            continue;
        }
        const std::string body = s.substr(ob, cb - ob);
        FusedConfig c;
        int wpb = 0, bal = 1;
        double ns = 0;
        const char *w = strstr(body.c_str(), "\"wpb\":");
        const char *b = strstr(body.c_str(), "\"balanced\":");
        const char *t = strstr(body.c_str(), "\"ns_per_ct\":");
        const char *tb = strstr(body.c_str(), "\"tile_below\":");
        unsigned tbv = 0;
        if (w && tb && sscanf(tb + 13, "%u", &tbv) == 1 && sscanf(w + 6, "%d", &wpb) == 1 && (wpb == 4 || wpb == 8)) {
            c.tile_below = tbv;
            c.wpb = wpb;
            if (b)
                sscanf(b + 11, "%d", &bal);
            if (t)
                sscanf(t + 12, "%lf", &ns);
            c.balanced = bal != 0;
            c.ns_per_ct = ns;
            c.tuned = true;
            out[key] = c;
        }
        pos = cb + 1;
    }
    return out;
}

static void save_cache(const std::map<std::string, FusedConfig> &m)
{
    const std::string p = cache_path();
    for (size_t i = 1; i < p.size(); i++)
        if (p[i] == '/') {
            std::string d = p.substr(0, i);
            mkdir(d.c_str(), 0755);
        }
    FILE *f = fopen(p.c_str(), "wb");
    if (!f)
        return;
    fprintf(f, "{\n");
    size_t i = 0;
    for (const auto &kv : m) {
        fprintf(f, "  \"%s\": {\"wpb\": %d, \"balanced\": %d, \"ns_per_ct\": %.3f, \"tile_below\": %u}%s\n",
                kv.first.c_str(), kv.second.wpb, kv.second.balanced ? 1 : 0, kv.second.ns_per_ct,
                kv.second.tile_below, ++i < m.size() ? "," : "");
    }
    fprintf(f, "}\n");
    fclose(f);
}

// A tuning for a given batch size is kept apart from the default one: which
// configuration wins depends on how a batch of that size fills whole rounds
// of the resident warps, not only on the kernel's steady-state rate.
static std::string cache_key(const cmd_engine *eng, int set, size_t sample_count)
{
    std::string k = std::string(eng->gpu_name) + "|" + std::to_string(set_info(set).id);
    if (sample_count)
        k += "|n=" + std::to_string(sample_count);
    return k;
}

}  // namespace cmd

using namespace cmd;

struct cmd_graph {
    cmd_engine *eng = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t *counter = nullptr;
    uint64_t kernels = 0;  // our kernels per replay
};

extern "C" {

int cmd_engine_fused_config(cmd_engine *eng, cmd_set set, int *wpb, int *balanced, double *ns_per_ct)
{
    if (!eng || !valid_set(set))
        return CMD_E_ARG;
    const FusedConfig &c = eng->fcfg[set];
    if (wpb)
        *wpb = c.wpb;
    if (balanced)
        *balanced = c.balanced ? 1 : 0;
    if (ns_per_ct)
        *ns_per_ct = c.ns_per_ct;
    return CMD_OK;
}

int cmd_engine_tile_below(cmd_engine *eng, cmd_set set, uint32_t *tile_below)
{
    if (!eng || !valid_set(set) || !tile_below)
        return CMD_E_ARG;
    *tile_below = eng->fcfg[set].tile_below;
    return CMD_OK;
}

int cmd_engine_set_fused_config(cmd_engine *eng, cmd_set set, int wpb, int balanced)
{
    if (!eng || !valid_set(set) || (wpb != 4 && wpb != 8))
        return CMD_E_ARG;
    std::lock_guard<std::mutex> lk(eng->mu);
    eng->fcfg[set].wpb = wpb;
    eng->fcfg[set].balanced = balanced != 0;
    eng->fcfg[set].tuned = false;
    return CMD_OK;
}

int cmd_tune(cmd_engine *eng, const cmd_key *key, size_t sample_count, int force)
{
    if (!eng || !key || key->eng != eng)
        return CMD_E_ARG;
    const int set = key->dev.set;
    const SetInfo si = set_info(set);
    cudaSetDevice(eng->device);
    auto cache = load_cache();
    const std::string ck = cache_key(eng, set, sample_count);
    if (!force) {
        auto it = cache.find(ck);
        if (it != cache.end()) {
            std::lock_guard<std::mutex> lk(eng->mu);
            eng->fcfg[set] = it->second;
            return CMD_OK;
        }
    }
    if (sample_count == 0)
        sample_count = (size_t)eng->num_sms * 256 * 3 + 1000;  // ~3 waves with a ragged tail
    std::lock_guard<std::mutex> lk(eng->mu);
    const size_t need = sample_count * si.ct + 256 + sample_count * si.nw * 4 + 256;
    int rc = eng->io.reserve(eng, need);
    if (rc)
        return rc;
    uint8_t *d_cts = static_cast<uint8_t *>(eng->io.ptr);
    uint32_t *d_err = reinterpret_cast<uint32_t *>(d_cts + (sample_count * si.ct + 255) / 256 * 256);
    if (!eng->tile_counter) {
        cudaError_t e = cudaMalloc(&eng->tile_counter, 256);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaMalloc(counter)");
    }
    cudaStream_t s = eng->stream;
    cudaError_t e = cudaMemsetAsync(d_cts, 0xA5, sample_count * si.ct, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "tune sample");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const FusedConfig saved = eng->fcfg[set];
    FusedConfig best = saved;
    double best_ns = 1e30;
    const int wpbs[2] = {8, 4};
    for (int wpb : wpbs) {
        for (int bal = 1; bal >= 0; bal--) {
            if (fused_smem(set, wpb) > smem_limit_bytes())
                continue;
            eng->fcfg[set].wpb = wpb;
            eng->fcfg[set].balanced = bal != 0;
            float total = 0;
            bool ok = true;
            for (int rep = 0; rep < 4 && ok; rep++) {
                cudaEventRecord(e0, s);
                ok = run_fused_counter(eng, key, d_cts, sample_count, d_err, nullptr, s, eng->tile_counter, nullptr, -1) == 0;
                cudaEventRecord(e1, s);
                if (cudaEventSynchronize(e1) != cudaSuccess)
                    ok = false;
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0)
                    total += ms;
            }
            if (!ok)
                continue;
            const double ns = total / 3 * 1e6 / (double)sample_count;
            if (ns < best_ns) {
                best_ns = ns;
                best.wpb = wpb;
                best.balanced = bal != 0;
            }
        }
    }
    if (best_ns >= 1e30) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        eng->fcfg[set] = saved;
        set_last_error("tuner: no candidate configuration ran");
        return CMD_E_CUDA;
    }
    eng->fcfg[set] = best;
    // Fused kernel (one warp per tile) against the tile kernels at growing
    // batch sizes: the tile kernels finish small batches sooner (their
    // Berlekamp-Massey runs on five warps, their FFTs on a warp per
    // ciphertext), the fused kernel does less work per ciphertext.
    best.tile_below = 0;
    const size_t sizes[] = {256, 1024, 4096, 16384, 65536};
    for (size_t n : sizes) {
        if (n > sample_count)
            break;
        auto timed = [&](bool tile) -> double {
            float total = 0;
            for (int rep = 0; rep < 3; rep++) {
                cudaEventRecord(e0, s);
                const int r = tile ? run_device(eng, key, CMD_PATH_TILE, d_cts, n, d_err, nullptr, s)
                                   : run_fused_counter(eng, key, d_cts, n, d_err, nullptr, s, eng->tile_counter,
                                                       nullptr, -1);
                cudaEventRecord(e1, s);
                if (r != CMD_OK || cudaEventSynchronize(e1) != cudaSuccess)
                    return 1e30;
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0)
                    total += ms;
            }
            return total / 2;
        };
        const double tf = timed(false), tt = timed(true);
        if (tt < tf)
            best.tile_below = (uint32_t)(2 * n);  // the tile kernels still win here
        else
            break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    best.tuned = true;
    best.ns_per_ct = best_ns;
    eng->fcfg[set] = best;
    cache[ck] = best;
    save_cache(cache);
    return CMD_OK;
}

int cmd_graph_capture(cmd_engine *eng, const cmd_key *key, cmd_path path, const uint8_t *d_cts, size_t count,
                      uint32_t *d_err, uint16_t *d_weight, cmd_graph **out)
{
    if (!eng || !key || key->eng != eng || !out || !count || !d_cts || !d_err || path < 0 || path > 2)
        return CMD_E_ARG;
    *out = nullptr;
    cudaSetDevice(eng->device);
    std::lock_guard<std::mutex> lk(eng->mu);
    cmd_graph *g = new cmd_graph();
    g->eng = eng;
    // Everything that may allocate or set function attributes happens before
    // the capture begins.
    int rc = CMD_OK;
    cudaError_t e = cudaSuccess;
    if (path == CMD_PATH_PLAIN) {
        rc = eng->scratch.reserve(eng, plain_scratch_bytes(key->dev.set, count));
    } else {
        e = cudaMalloc(&g->counter, 256);
        if (e == cudaSuccess)
            e = fused_prepare(eng, key->dev.set);
    }
    if (rc || e != cudaSuccess) {
        if (g->counter)
            cudaFree(g->counter);
        delete g;
        return rc ? rc : cuda_fail(e, "graph setup");
    }
    cudaStream_t cs;
    if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) {
        cudaFree(g->counter);
        delete g;
        return cuda_fail(e, "cudaStreamCreate(capture)");
    }
    const uint64_t before = eng->launches.load();
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        if (path == CMD_PATH_PLAIN)
            rc = run_device(eng, key, path, d_cts, count, d_err, d_weight, cs);
        else
            rc = run_fused_counter(eng, key, d_cts, count, d_err, d_weight, cs, g->counter, nullptr, -1);
        cudaGraph_t graph = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if (rc == CMD_OK && e2 != cudaSuccess)
            rc = cuda_fail(e2, "cudaStreamEndCapture");
        g->graph = graph;
    } else {
        rc = cuda_fail(e, "cudaStreamBeginCapture");
    }
    g->kernels = eng->launches.load() - before;
    eng->launches.fetch_sub(g->kernels);  // captured, not launched
    cudaStreamDestroy(cs);
    if (rc == CMD_OK && (e = cudaGraphInstantiate(&g->exec, g->graph, 0)) != cudaSuccess)
        rc = cuda_fail(e, "cudaGraphInstantiate");
    if (rc != CMD_OK) {
        if (g->exec)
            cudaGraphExecDestroy(g->exec);
        if (g->graph)
            cudaGraphDestroy(g->graph);
        if (g->counter)
            cudaFree(g->counter);
        delete g;
        return rc;
    }
    *out = g;
    return CMD_OK;
}

int cmd_graph_launch(cmd_graph *g, void *stream)
{
    if (!g)
        return CMD_E_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : g->eng->stream;
    cudaError_t e = cudaGraphLaunch(g->exec, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGraphLaunch");
    g->eng->launches.fetch_add(g->kernels);
    return CMD_OK;
}

void cmd_graph_destroy(cmd_graph *g)
{
    if (!g)
        return;
    if (g->exec)
        cudaGraphExecDestroy(g->exec);
    if (g->graph)
        cudaGraphDestroy(g->graph);
    if (g->counter)
        cudaFree(g->counter);
    delete g;
}

}  // extern "C"
