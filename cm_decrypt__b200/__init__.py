"""B200-native batched Classic McEliece decryption engine.

Drop-in for the decrypt path of somesh-vas/CM_Decrypt_: same sk_<set>.bin /
ct_<set>.bin inputs, same errorstream0_<set>.bin text, bit-exact with the
reference CPU/ decoder for the five parameter sets.  All decoding runs in the
CUDA kernels of libcmd_b200.so (sm_100a); this module is a thin ctypes
front-end over its C ABI (include/cmd_b200.h).  There is no CPU fallback: on a
machine without a B200 the compute calls raise CmdError.

The names mirror the reference's decoder interface (CPU/include/common/
root.h, bm.h): ``Key`` replaces initialisation() + support_gen() +
compute_inverses(); ``synd``, ``bm`` and ``root`` are the per-stage hooks;
``decrypt`` is the per-ciphertext loop of decrypt.c run as one batch;
``errorstream`` / ``decrypt_files`` are write_error_positions and the CLI.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libcmd_b200.so")
CLI_PATH = os.path.join(PKG_DIR, "cmd_decrypt")

SETS = (348864, 460896, 6688128, 6960119, 8192128)
SET_INDEX = {s: i for i, s in enumerate(SETS)}

# Status codes (include/cmd_b200.h); 0/-1/-4 are the reference's KAT_* codes.
CMD_OK, CMD_E_FILE, CMD_E_ARG, CMD_E_CUDA = 0, -1, -4, -5
CMD_E_NOMEM, CMD_E_BUDGET, CMD_E_BUSY, CMD_E_TIMEOUT, CMD_E_NODEVICE = -6, -7, -8, -9, -10
PATHS = {"auto": 0, "plain": 1, "fused": 2, "tile": 3}


class CmdError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed with status {code}: {_last_error()}")
        self.code = code


class _SetInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in
                ("set_id", "m", "n", "t", "ct_bytes", "sk_bytes", "sb", "err_bytes", "err_words")]


@dataclass(frozen=True)
class SetInfo:
    set_id: int
    m: int
    n: int
    t: int
    ct_bytes: int
    sk_bytes: int
    sb: int
    err_bytes: int
    err_words: int


class ServerConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in
                ("max_batch", "slots", "max_wait_us", "queue_capacity", "fused_threshold", "record_completions")]


class Completion(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("status", ctypes.c_int32), ("weight", ctypes.c_uint16),
                ("reserved", ctypes.c_uint16), ("latency_ns", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("submitted", "completed", "refused", "batches", "fused_batches", "resident_keys")] + \
               [(n, ctypes.c_double) for n in
                ("mean_batch", "p50_us", "p99_us", "max_us", "mean_us", "decaps_per_s", "offered_per_s",
                 "gpu_p50_us", "gpu_p99_us", "wait_p50_us", "wait_p99_us", "dispatch_busy", "complete_busy",
                 "mean_inflight")]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib: ctypes.CDLL | None = None
_vp, _sz, _u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64
_i32 = ctypes.c_int


def lib() -> ctypes.CDLL:
    """Loads libcmd_b200.so (built in-tree by cm_decrypt__b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} missing: run `python -m cm_decrypt__b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "cmd_last_error": (ctypes.c_char_p, []),
        "cmd_set_info_get": (_i32, [_i32, ctypes.POINTER(_SetInfo)]),
        "cmd_set_from_name": (_i32, [ctypes.c_char_p, ctypes.POINTER(_i32)]),
        "cmd_engine_create": (_i32, [_i32, _sz, ctypes.POINTER(_vp)]),
        "cmd_engine_destroy": (None, [_vp]),
        "cmd_engine_memory": (_i32, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz)]),
        "cmd_engine_launch_count": (_u64, [_vp]),
        "cmd_key_expand": (_i32, [_vp, _i32, _vp, _sz, ctypes.POINTER(_vp)]),
        "cmd_key_free": (None, [_vp]),
        "cmd_key_set": (_i32, [_vp, ctypes.POINTER(_i32)]),
        "cmd_key_device_bytes": (_sz, [_vp]),
        "cmd_key_support": (_i32, [_vp, _vp, _sz]),
        "cmd_key_goppa": (_i32, [_vp, _vp, _sz]),
        "cmd_key_synd_table": (_i32, [_vp, _vp, _sz]),
        "cmd_decrypt_batch": (_i32, [_vp, _vp, _i32, _vp, _sz, _vp, _vp]),
        "cmd_decrypt_device": (_i32, [_vp, _vp, _i32, _vp, _sz, _vp, _vp, _vp]),
        "cmd_decrypt_mixed_device": (_i32, [_vp, _vp, _sz, _vp, _vp, _vp, _sz, _vp, _vp, _vp, _vp]),
        "cmd_decrypt_plain_noalloc": (_i32, [_vp, _vp, _sz, _vp, _vp, _vp]),
        "cmd_stage_synd": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp]),
        "cmd_stage_synd_fft": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp]),
        "cmd_stage_bm": (_i32, [_vp, _i32, _vp, _sz, _vp, _vp]),
        "cmd_stage_root": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp, _vp]),
        "cmd_stage_root_images": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp]),
        "cmd_errorstream_format": (_i32, [_i32, _vp, _sz, _vp, _sz, ctypes.POINTER(_sz)]),
        "cmd_errorstream_write": (_i32, [_i32, _vp, _sz, ctypes.c_char_p, _i32]),
        "cmd_key_prepare_decap": (_i32, [_vp, _vp]),
        "cmd_kem_decap": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp]),
        "cmd_kem_keypair": (_i32, [_vp, _i32, _vp, _vp, _vp, _vp]),
        "cmd_kem_keypair_batch": (_i32, [_vp, _i32, _vp, _sz, _vp, _vp, _vp, ctypes.c_uint32]),
        "cmd_kem_decap_device": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp, _vp]),
        "cmd_pubkey_columns": (_i32, [_vp, _vp, _sz, ctypes.POINTER(_sz)]),
        "cmd_decrypt_positions": (_i32, [_vp, _vp, _vp, _sz, _vp]),
        "cmd_decrypt_positions_device": (_i32, [_vp, _vp, _vp, _sz, _vp, _vp]),
        "cmd_positions_format": (_i32, [_i32, _vp, _sz, _vp, _sz, ctypes.POINTER(_sz)]),
        "cmd_positions_write": (_i32, [_i32, _vp, _sz, ctypes.c_char_p, _i32]),
        "cmd_positions_to_errorstream": (_i32, [ctypes.c_char_p, ctypes.c_char_p]),
        "cmd_decrypt_files_binary": (_i32, [_vp, _i32, ctypes.c_char_p, ctypes.c_char_p, _sz, ctypes.c_char_p,
                                            ctypes.POINTER(ctypes.c_double)]),
        "cmd_decrypt_files": (_i32, [_vp, _i32, ctypes.c_char_p, ctypes.c_char_p, _sz, ctypes.c_char_p, _i32,
                                     ctypes.POINTER(ctypes.c_double)]),
        "cmd_bench_int_peak": (_i32, [_vp, ctypes.POINTER(ctypes.c_double)]),
        "cmd_tune": (_i32, [_vp, _vp, _sz, _i32]),
        "cmd_engine_fused_config": (_i32, [_vp, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                                           ctypes.POINTER(ctypes.c_double)]),
        "cmd_engine_tile_below": (_i32, [_vp, _i32, ctypes.POINTER(ctypes.c_uint32)]),
        "cmd_engine_set_fused_config": (_i32, [_vp, _i32, _i32, _i32]),
        "cmd_graph_capture": (_i32, [_vp, _vp, _i32, _vp, _sz, _vp, _vp, ctypes.POINTER(_vp)]),
        "cmd_graph_launch": (_i32, [_vp, _vp]),
        "cmd_graph_destroy": (None, [_vp]),
        "cmd_server_create": (_i32, [_vp, ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]),
        "cmd_server_destroy": (None, [_vp]),
        "cmd_server_add_key": (_i32, [_vp, _i32, _vp, _sz, ctypes.POINTER(ctypes.c_uint32)]),
        "cmd_server_submit": (_i32, [_vp, ctypes.c_uint32, _vp, _vp, _u64]),
        "cmd_server_submit_many": (_i32, [_vp, _sz, _vp, _vp, _sz, _vp, _sz, _vp, ctypes.POINTER(_sz)]),
        "cmd_server_register_rows": (_i32, [_vp, _vp, _sz]),
        "cmd_server_poll": (_i32, [_vp, ctypes.POINTER(Completion), _sz, ctypes.POINTER(_sz), ctypes.c_uint32]),
        "cmd_server_drain": (_i32, [_vp, ctypes.c_uint32]),
        "cmd_server_stats_get": (_i32, [_vp, ctypes.POINTER(ServerStats), _i32]),
        "cmd_server_loadgen": (_i32, [_vp, _vp, _vp, _sz, _vp, _sz, _sz, ctypes.c_double, ctypes.c_double, _u64,
                                      ctypes.POINTER(ServerStats)]),
        "cmd_synth_key": (_i32, [_i32, _vp, _u64, _vp]),
        "cmd_synth_pubkey": (_i32, [_i32, _vp, ctypes.POINTER(_vp)]),
        "cmd_synth_pubkey_free": (None, [_vp]),
        "cmd_synth_ciphertexts": (_i32, [_vp, _u64, _sz, ctypes.c_uint32, _vp, _vp, _vp, _i32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _last_error() -> str:
    try:
        return (lib().cmd_last_error() or b"").decode()
    except Exception:  # pragma: no cover - only when the library is absent
        return ""


def _check(code: int, what: str) -> None:
    if code != CMD_OK:
        raise CmdError(code, what)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def set_index(set_id: int) -> int:
    if set_id in SET_INDEX:
        return SET_INDEX[set_id]
    if 0 <= set_id < len(SETS):
        return set_id
    raise ValueError(f"unknown parameter set {set_id}")


def set_info(set_id: int) -> SetInfo:
    info = _SetInfo()
    _check(lib().cmd_set_info_get(set_index(set_id), ctypes.byref(info)), "cmd_set_info_get")
    return SetInfo(*[getattr(info, f) for f, _ in _SetInfo._fields_])


class Engine:
    """One engine per GPU; owns the stream, scratch and the HBM budget."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = _vp()
        _check(lib().cmd_engine_create(device, hbm_budget, ctypes.byref(h)), "cmd_engine_create")
        self.handle = h

    def close(self) -> None:
        if self.handle:
            lib().cmd_engine_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def memory(self) -> tuple[int, int]:
        used, budget = _sz(), _sz()
        _check(lib().cmd_engine_memory(self.handle, ctypes.byref(used), ctypes.byref(budget)), "memory")
        return used.value, budget.value

    def launch_count(self) -> int:
        return int(lib().cmd_engine_launch_count(self.handle))

    def int_peak(self) -> float:
        """Measured lop3.b32 lane-operations per second (int-ALU roofline)."""
        v = ctypes.c_double()
        _check(lib().cmd_bench_int_peak(self.handle, ctypes.byref(v)), "cmd_bench_int_peak")
        return v.value


class Key:
    """Device-resident expanded secret key (support, 1/g(L)^2, tables)."""

    def __init__(self, engine: Engine, set_id: int, sk: bytes):
        self.engine = engine
        self.info = set_info(set_id)
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        h = _vp()
        _check(lib().cmd_key_expand(engine.handle, set_index(set_id), _ptr(skb), skb.size, ctypes.byref(h)),
               "cmd_key_expand")
        self.handle = h

    def free(self) -> None:
        if self.handle:
            lib().cmd_key_free(self.handle)
            self.handle = None

    def device_bytes(self) -> int:
        return int(lib().cmd_key_device_bytes(self.handle))

    def support(self) -> np.ndarray:
        out = np.zeros(self.info.n, np.uint16)
        _check(lib().cmd_key_support(self.handle, _ptr(out), out.size), "cmd_key_support")
        return out

    def goppa(self) -> np.ndarray:
        out = np.zeros(self.info.t + 1, np.uint16)
        _check(lib().cmd_key_goppa(self.handle, _ptr(out), out.size), "cmd_key_goppa")
        return out

    def synd_table(self) -> np.ndarray:
        out = np.zeros((self.info.sb, 2 * self.info.t), np.uint16)
        _check(lib().cmd_key_synd_table(self.handle, _ptr(out), out.size), "cmd_key_synd_table")
        return out


def decrypt(engine: Engine, key: Key, cts, path: str = "auto") -> tuple[np.ndarray, np.ndarray]:
    """Host batch: cts uint8 [count, ct_bytes] -> (err uint8 [count, n/8], weight uint16 [count])."""
    info = key.info
    c = np.ascontiguousarray(np.frombuffer(bytes(cts), np.uint8) if isinstance(cts, (bytes, bytearray))
                             else cts, np.uint8).reshape(-1, info.ct_bytes)
    err = np.zeros((c.shape[0], info.err_bytes), np.uint8)
    w = np.zeros(c.shape[0], np.uint16)
    _check(lib().cmd_decrypt_batch(engine.handle, key.handle, PATHS[path], _ptr(c), c.shape[0], _ptr(err), _ptr(w)),
           "cmd_decrypt_batch")
    return err, w


def decrypt_into(engine: Engine, key: Key, cts: np.ndarray, err: np.ndarray, weight: np.ndarray | None = None,
                 path: str = "auto") -> None:
    """Host batch into caller buffers (pinned buffers make the copies DMA)."""
    info = key.info
    assert cts.dtype == np.uint8 and cts.flags.c_contiguous and cts.size % info.ct_bytes == 0
    count = cts.size // info.ct_bytes
    assert err.dtype == np.uint8 and err.flags.c_contiguous and err.size == count * info.err_bytes
    wp = 0
    if weight is not None:
        assert weight.dtype == np.uint16 and weight.size == count
        wp = _ptr(weight)
    _check(lib().cmd_decrypt_batch(engine.handle, key.handle, PATHS[path], _ptr(cts), count, _ptr(err), wp or None),
           "cmd_decrypt_batch")


def decrypt_device(engine: Engine, key: Key, d_cts: int, count: int, d_err: int, d_weight: int = 0,
                   stream: int = 0, path: str = "auto") -> None:
    """Device pointers (e.g. torch tensor data_ptr()); asynchronous on `stream`."""
    _check(lib().cmd_decrypt_device(engine.handle, key.handle, PATHS[path], d_cts, count, d_err,
                                    d_weight or None, stream or None), "cmd_decrypt_device")


def decrypt_mixed_device(engine: Engine, keys: list[Key], key_idx: np.ndarray, d_cts: int, ct_off: np.ndarray,
                         d_err: int, err_off: np.ndarray, d_weight: int = 0, stream: int = 0) -> None:
    arr = (_vp * len(keys))(*[k.handle for k in keys])
    ki = np.ascontiguousarray(key_idx, np.uint32)
    co = np.ascontiguousarray(ct_off, np.uint64)
    eo = np.ascontiguousarray(err_off, np.uint64)
    _check(lib().cmd_decrypt_mixed_device(engine.handle, arr, len(keys), _ptr(ki), d_cts, _ptr(co), ki.size, d_err,
                                          _ptr(eo), d_weight or None, stream or None), "cmd_decrypt_mixed_device")


def tune(engine: Engine, key: Key, sample_count: int = 0, force: bool = False) -> dict:
    """Autotunes the fused kernel for key's set; returns the chosen config."""
    _check(lib().cmd_tune(engine.handle, key.handle, sample_count, int(force)), "cmd_tune")
    return fused_config(engine, key.info.set_id)


def fused_config(engine: Engine, set_id: int) -> dict:
    wpb, bal, ns = _i32(), _i32(), ctypes.c_double()
    _check(lib().cmd_engine_fused_config(engine.handle, set_index(set_id), ctypes.byref(wpb), ctypes.byref(bal),
                                         ctypes.byref(ns)), "cmd_engine_fused_config")
    tb = ctypes.c_uint32()
    _check(lib().cmd_engine_tile_below(engine.handle, set_index(set_id), ctypes.byref(tb)), "cmd_engine_tile_below")
    return {"wpb": wpb.value, "balanced": bool(bal.value), "ns_per_ct": ns.value, "tile_below": tb.value}


def set_fused_config(engine: Engine, set_id: int, wpb: int, balanced: bool = True) -> None:
    _check(lib().cmd_engine_set_fused_config(engine.handle, set_index(set_id), wpb, int(balanced)),
           "cmd_engine_set_fused_config")


class Graph:
    """A decrypt over fixed device buffers, captured once, replayed many times."""

    def __init__(self, engine: Engine, key: Key, d_cts: int, count: int, d_err: int, d_weight: int = 0,
                 path: str = "fused"):
        h = _vp()
        _check(lib().cmd_graph_capture(engine.handle, key.handle, PATHS[path], d_cts, count, d_err,
                                       d_weight or None, ctypes.byref(h)), "cmd_graph_capture")
        self.handle = h

    def launch(self, stream: int = 0) -> None:
        _check(lib().cmd_graph_launch(self.handle, stream or None), "cmd_graph_launch")

    def close(self) -> None:
        if self.handle:
            lib().cmd_graph_destroy(self.handle)
            self.handle = None


class Server:
    """Continuous-batching decapsulation server (see cmd_server_* in the header)."""

    def __init__(self, engine: Engine, max_batch: int = 2048, slots: int = 4, max_wait_us: int = 200,
                 queue_capacity: int = 1 << 20, fused_threshold: int = 0, record_completions: bool = True):
        cfg = ServerConfig(max_batch, slots, max_wait_us, queue_capacity, fused_threshold, int(record_completions))
        h = _vp()
        _check(lib().cmd_server_create(engine.handle, ctypes.byref(cfg), ctypes.byref(h)), "cmd_server_create")
        self.handle = h
        self.key_sets: list[int] = []
        self._rows: list[np.ndarray] = []  # registered row memory, kept alive until close()

    def close(self) -> None:
        if self.handle:
            lib().cmd_server_destroy(self.handle)
            self.handle = None
        self._rows = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_key(self, set_id: int, sk: bytes) -> int:
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        kid = ctypes.c_uint32()
        _check(lib().cmd_server_add_key(self.handle, set_index(set_id), _ptr(skb), skb.size, ctypes.byref(kid)),
               "cmd_server_add_key")
        self.key_sets.append(set_id)
        return kid.value

    def register_rows(self, rows: np.ndarray) -> None:
        """Result rows inside `rows` (a C-contiguous array, kept alive by the
        server until close()) are stored there by the GPU itself on the
        latency kernels' path (cmd_server_register_rows)."""
        if not rows.flags.c_contiguous:
            raise ValueError("register_rows needs a C-contiguous array")
        _check(lib().cmd_server_register_rows(self.handle, _ptr(rows), rows.nbytes), "cmd_server_register_rows")
        self._rows.append(rows)

    def submit(self, key_id: int, ct: np.ndarray, err_out: np.ndarray | None, tag: int) -> int:
        """Returns CMD_OK or CMD_E_BUSY; err_out must stay alive until completion."""
        rc = lib().cmd_server_submit(self.handle, key_id, _ptr(ct), _ptr(err_out) if err_out is not None else None,
                                     tag)
        if rc not in (CMD_OK, CMD_E_BUSY):
            raise CmdError(rc, "cmd_server_submit")
        return rc

    def submit_many(self, key_ids: np.ndarray, cts: np.ndarray, err_out: np.ndarray | None,
                    tags: np.ndarray | None = None) -> int:
        """Queues len(key_ids) requests under one lock (cts rows, err_out rows);
        returns how many were accepted.  err_out must stay alive until completion."""
        ki = np.ascontiguousarray(key_ids, np.uint32)
        c = np.ascontiguousarray(cts, np.uint8)
        tg = None if tags is None else np.ascontiguousarray(tags, np.uint64)
        acc = _sz()
        rc = lib().cmd_server_submit_many(self.handle, ki.size, _ptr(ki), _ptr(c), c.shape[1],
                                          _ptr(err_out) if err_out is not None else None,
                                          err_out.shape[1] if err_out is not None else 0,
                                          _ptr(tg) if tg is not None else None, ctypes.byref(acc))
        if rc not in (CMD_OK, CMD_E_BUSY):
            raise CmdError(rc, "cmd_server_submit_many")
        return acc.value

    def poll(self, max_n: int = 4096, timeout_us: int = 0) -> list[tuple[int, int, int, int]]:
        buf = (Completion * max_n)()
        n = _sz()
        _check(lib().cmd_server_poll(self.handle, buf, max_n, ctypes.byref(n), timeout_us), "cmd_server_poll")
        return [(c.tag, c.status, c.weight, c.latency_ns) for c in buf[: n.value]]

    def drain(self, timeout_ms: int = 60000) -> None:
        _check(lib().cmd_server_drain(self.handle, timeout_ms), "cmd_server_drain")

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        _check(lib().cmd_server_stats_get(self.handle, ctypes.byref(st), int(reset)), "cmd_server_stats_get")
        return st.as_dict()

    def loadgen(self, key_ids: np.ndarray, cts: np.ndarray, err_pool: np.ndarray | None, rate: float,
                seconds: float, seed: int = 0x5EED) -> dict:
        ki = np.ascontiguousarray(key_ids, np.uint32)
        c = np.ascontiguousarray(cts, np.uint8)
        st = ServerStats()
        _check(lib().cmd_server_loadgen(self.handle, _ptr(ki), _ptr(c), c.shape[1],
                                        _ptr(err_pool) if err_pool is not None else None,
                                        err_pool.shape[1] if err_pool is not None else 0, ki.size, rate, seconds,
                                        seed, ctypes.byref(st)), "cmd_server_loadgen")
        return st.as_dict()


# ---- per-stage hooks (device pointers) -----------------------------------
def synd(engine: Engine, key: Key, d_cts: int, count: int, d_synd: int, stream: int = 0) -> None:
    _check(lib().cmd_stage_synd(engine.handle, key.handle, d_cts, count, d_synd, stream or None), "synd")


def synd_fft(engine: Engine, key: Key, d_cts: int, count: int, d_synd: int, stream: int = 0) -> None:
    """synd() by the serving path's transposed additive FFT (no syndrome table)."""
    _check(lib().cmd_stage_synd_fft(engine.handle, key.handle, d_cts, count, d_synd, stream or None), "synd_fft")


def bm(engine: Engine, set_id: int, d_synd: int, count: int, d_loc: int, stream: int = 0) -> None:
    _check(lib().cmd_stage_bm(engine.handle, set_index(set_id), d_synd, count, d_loc, stream or None), "bm")


def root(engine: Engine, key: Key, d_loc: int, count: int, d_err: int, d_weight: int = 0, stream: int = 0) -> None:
    _check(lib().cmd_stage_root(engine.handle, key.handle, d_loc, count, d_err, d_weight or None, stream or None),
           "root")


def root_images(engine: Engine, key: Key, d_loc: int, count: int, d_images: int, stream: int = 0) -> None:
    _check(lib().cmd_stage_root_images(engine.handle, key.handle, d_loc, count, d_images, stream or None),
           "root_images")


# ---- errorstream / file contract -------------------------------------------
def errorstream(set_id: int, err: np.ndarray) -> bytes:
    info = set_info(set_id)
    e = np.ascontiguousarray(err, np.uint8).reshape(-1, info.err_bytes)
    need = _sz()
    lib().cmd_errorstream_format(set_index(set_id), _ptr(e), e.shape[0], None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(need.value + 1)
    _check(lib().cmd_errorstream_format(set_index(set_id), _ptr(e), e.shape[0], buf, need.value + 1,
                                        ctypes.byref(need)), "cmd_errorstream_format")
    return buf.raw[:need.value]


def write_errorstream(set_id: int, err: np.ndarray, path: str, append: bool = False) -> None:
    info = set_info(set_id)
    e = np.ascontiguousarray(err, np.uint8).reshape(-1, info.err_bytes)
    _check(lib().cmd_errorstream_write(set_index(set_id), _ptr(e), e.shape[0], path.encode(), int(append)),
           "cmd_errorstream_write")


def decrypt_files(engine: Engine, set_id: int, sk_path: str, ct_path: str, katnum: int, out_path: str,
                  path: str = "auto") -> float:
    secs = ctypes.c_double()
    _check(lib().cmd_decrypt_files(engine.handle, set_index(set_id), sk_path.encode(), ct_path.encode(), katnum,
                                   out_path.encode(), PATHS[path], ctypes.byref(secs)), "cmd_decrypt_files")
    return secs.value


# ---- KEM decapsulation --------------------------------------------------------
def pk_bytes(set_id: int) -> int:
    """Public-key bytes: mt rows of (n - mt + 7)/8 bytes (pk_gen.c:145-146)."""
    info = set_info(set_id)
    mt = info.m * info.t
    return mt * ((info.n - mt + 7) // 8)


def kem_keypair(engine: Engine, set_id: int, seed: bytes) -> tuple[bytes, bytes, int]:
    """crypto_kem_keypair with randombytes() yielding `seed` (32 bytes), on
    the GPU.  Returns (pk, sk, attempts)."""
    seed = bytes(seed)
    if len(seed) != 32:
        raise ValueError("seed must be 32 bytes")
    info = set_info(set_id)
    pk = np.zeros(pk_bytes(set_id), np.uint8)
    sk = np.zeros(info.sk_bytes, np.uint8)
    att = ctypes.c_uint32()
    sb = np.frombuffer(seed, np.uint8).copy()
    _check(lib().cmd_kem_keypair(engine.handle, set_index(set_id), _ptr(sb), _ptr(pk), _ptr(sk), ctypes.byref(att)),
           "cmd_kem_keypair")
    return pk.tobytes(), sk.tobytes(), att.value


def kem_keypair_batch(engine: Engine, set_id: int, seeds: np.ndarray, max_attempts: int = 0,
                      pk_out: np.ndarray | None = None,
                      sk_out: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Key pairs for a batch of 32-byte seeds: (pk uint8 [count, pk_bytes],
    sk uint8 [count, sk_bytes], attempts uint32 [count]).  pk_out / sk_out,
    when given, are written in place (e.g. pinned host buffers, which make the
    result copies faster)."""
    sd = np.ascontiguousarray(seeds, np.uint8).reshape(-1, 32)
    info = set_info(set_id)
    shape_pk, shape_sk = (sd.shape[0], pk_bytes(set_id)), (sd.shape[0], info.sk_bytes)
    for name, arr, shape in (("pk_out", pk_out, shape_pk), ("sk_out", sk_out, shape_sk)):
        if arr is not None and (arr.dtype != np.uint8 or arr.shape != shape or not arr.flags.c_contiguous):
            raise ValueError(f"{name} must be a C-contiguous uint8 array of shape {shape}")
    pk = pk_out if pk_out is not None else np.zeros(shape_pk, np.uint8)
    sk = sk_out if sk_out is not None else np.zeros(shape_sk, np.uint8)
    att = np.zeros(sd.shape[0], np.uint32)
    _check(lib().cmd_kem_keypair_batch(engine.handle, set_index(set_id), _ptr(sd), sd.shape[0], _ptr(pk), _ptr(sk),
                                       _ptr(att), max_attempts), "cmd_kem_keypair_batch")
    return pk, sk, att


def prepare_decap(engine: Engine, key: Key) -> None:
    """Derives the key's public key (host) and keeps it on the device."""
    _check(lib().cmd_key_prepare_decap(engine.handle, key.handle), "cmd_key_prepare_decap")


def kem_decap(engine: Engine, key: Key, cts: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Host buffers -> (keys uint8 [count, 32], accept uint8 [count])."""
    info = key.info
    c = np.ascontiguousarray(cts, np.uint8).reshape(-1, info.ct_bytes)
    keys = np.zeros((c.shape[0], 32), np.uint8)
    acc = np.zeros(c.shape[0], np.uint8)
    _check(lib().cmd_kem_decap(engine.handle, key.handle, _ptr(c), c.shape[0], _ptr(keys), _ptr(acc)),
           "cmd_kem_decap")
    return keys, acc


def kem_decap_device(engine: Engine, key: Key, d_cts: int, count: int, d_keys: int, d_accept: int = 0,
                     stream: int = 0) -> None:
    _check(lib().cmd_kem_decap_device(engine.handle, key.handle, d_cts, count, d_keys, d_accept or None,
                                      stream or None), "cmd_kem_decap_device")


# ---- error positions and the binary errorstream ------------------------------
def decrypt_positions(engine: Engine, key: Key, cts: np.ndarray) -> np.ndarray:
    """Host buffers -> uint16 [count, t+1]: weight, positions ascending, 0xFFFF."""
    info = key.info
    c = np.ascontiguousarray(cts, np.uint8).reshape(-1, info.ct_bytes)
    out = np.zeros((c.shape[0], info.t + 1), np.uint16)
    _check(lib().cmd_decrypt_positions(engine.handle, key.handle, _ptr(c), c.shape[0], _ptr(out)),
           "cmd_decrypt_positions")
    return out


def decrypt_positions_device(engine: Engine, key: Key, d_cts: int, count: int, d_pos: int, stream: int = 0) -> None:
    _check(lib().cmd_decrypt_positions_device(engine.handle, key.handle, d_cts, count, d_pos, stream or None),
           "cmd_decrypt_positions_device")


def positions_text(set_id: int, pos: np.ndarray) -> bytes:
    info = set_info(set_id)
    p = np.ascontiguousarray(pos, np.uint16).reshape(-1, info.t + 1)
    need = _sz()
    lib().cmd_positions_format(set_index(set_id), _ptr(p), p.shape[0], None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(need.value + 1)
    _check(lib().cmd_positions_format(set_index(set_id), _ptr(p), p.shape[0], buf, need.value + 1,
                                      ctypes.byref(need)), "cmd_positions_format")
    return buf.raw[:need.value]


def write_positions(set_id: int, pos: np.ndarray, path: str, append: bool = False) -> None:
    info = set_info(set_id)
    p = np.ascontiguousarray(pos, np.uint16).reshape(-1, info.t + 1)
    _check(lib().cmd_positions_write(set_index(set_id), _ptr(p), p.shape[0], path.encode(), int(append)),
           "cmd_positions_write")


def positions_to_errorstream(binary_path: str, text_path: str) -> None:
    _check(lib().cmd_positions_to_errorstream(binary_path.encode(), text_path.encode()),
           "cmd_positions_to_errorstream")


def decrypt_files_binary(engine: Engine, set_id: int, sk_path: str, ct_path: str, katnum: int,
                         out_path: str) -> float:
    secs = ctypes.c_double()
    _check(lib().cmd_decrypt_files_binary(engine.handle, set_index(set_id), sk_path.encode(), ct_path.encode(),
                                          katnum, out_path.encode(), ctypes.byref(secs)), "cmd_decrypt_files_binary")
    return secs.value


def positions_from_errors(set_id: int, err: np.ndarray) -> np.ndarray:
    """Reference conversion (host, numpy): packed error vectors -> positions rows."""
    info = set_info(set_id)
    e = np.ascontiguousarray(err, np.uint8).reshape(-1, info.err_bytes)
    bits = np.unpackbits(e, axis=1, bitorder="little")
    out = np.full((e.shape[0], info.t + 1), 0xFFFF, np.uint16)
    for r in range(e.shape[0]):
        idx = np.nonzero(bits[r])[0]
        out[r, 0] = idx.size
        out[r, 1: 1 + min(idx.size, info.t)] = idx[: info.t]
    return out


# ---- synthetic workloads -----------------------------------------------------
def synth_key(set_id: int, base_sk: bytes, seed: int) -> bytes:
    info = set_info(set_id)
    base = np.frombuffer(bytes(base_sk), np.uint8).copy()
    out = np.zeros(info.sk_bytes, np.uint8)
    _check(lib().cmd_synth_key(set_index(set_id), _ptr(base), seed, _ptr(out)), "cmd_synth_key")
    return out.tobytes()


class PubKey:
    """Systematic parity-check data for encrypting synthetic ciphertexts."""

    def __init__(self, set_id: int, sk: bytes):
        self.info = set_info(set_id)
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        h = _vp()
        _check(lib().cmd_synth_pubkey(set_index(set_id), _ptr(skb), ctypes.byref(h)), "cmd_synth_pubkey")
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.cmd_synth_pubkey_free(self.handle)
            self.handle = None

    def ciphertexts(self, seed: int, count: int, malformed_permille: int = 0, nthreads: int = 0):
        """-> (cts uint8 [count, ct_bytes], planted err uint8 [count, n/8], valid uint8 [count])."""
        info = self.info
        cts = np.zeros((count, info.ct_bytes), np.uint8)
        err = np.zeros((count, info.err_bytes), np.uint8)
        valid = np.zeros(count, np.uint8)
        nt = nthreads or min(32, os.cpu_count() or 1)
        _check(lib().cmd_synth_ciphertexts(self.handle, seed, count, malformed_permille, _ptr(cts), _ptr(err),
                                           _ptr(valid), nt), "cmd_synth_ciphertexts")
        return cts, err, valid

    def columns(self) -> np.ndarray:
        """The T block of [I | T]: uint64 [n - mt, words]; bit r of column i = T[r, i]."""
        info = self.info
        w = _sz()
        _check(lib().cmd_pubkey_columns(self.handle, None, 0, ctypes.byref(w)), "cmd_pubkey_columns")
        out = np.zeros((info.n - info.m * info.t, w.value), np.uint64)
        _check(lib().cmd_pubkey_columns(self.handle, _ptr(out), out.size, ctypes.byref(w)), "cmd_pubkey_columns")
        return out


def cuda_available() -> bool:
    """True when a CUDA device the engine can drive is present."""
    try:
        e = Engine()
    except (CmdError, FileNotFoundError, OSError):
        return False
    e.close()
    return True
