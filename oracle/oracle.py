"""ctypes front-end to the two CPU checkers in this directory.

TEST INFRASTRUCTURE ONLY.  ``Oracle`` wraps liboracle.so (the C restatement
of the reference decrypt path, cmd_oracle.c); ``RefLib`` wraps
_ref/libref_<set>.so (the reference's own CPU/ sources behind ref_harness.c).
Only tests/, the smoke entry point and bench.py's CPU-baseline leg use them.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SETS = (348864, 460896, 6688128, 6960119, 8192128)

_u16p = ctypes.POINTER(ctypes.c_uint16)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _ptr(a: np.ndarray, typ):
    return a.ctypes.data_as(typ)


class Params(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int) for name in
                ("set_id", "m", "n", "t", "ct_bytes", "sk_bytes", "sb", "cond_bytes")]


def reference_dir() -> str:
    """The reference tree: $CMD_REFERENCE_DIR, else a checkout named
    `reference` beside this repository; "" when neither exists."""
    env = os.environ.get("CMD_REFERENCE_DIR", "")
    if env:
        return env
    beside = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
    return beside if os.path.isdir(os.path.join(beside, "CPU")) else ""


def build(with_reference: bool | None = None, ref_dir: str | None = None) -> None:
    """Compile liboracle.so and, when the reference tree is present
    (`ref_dir`, else reference_dir()), _ref/.  with_reference=True requires
    it."""
    ref_dir = ref_dir or reference_dir()
    targets = ["oracle"]
    have = bool(ref_dir) and os.path.isdir(os.path.join(ref_dir, "CPU"))
    if with_reference and not have:
        raise FileNotFoundError("the reference tree: pass ref_dir or set CMD_REFERENCE_DIR")
    if with_reference or (with_reference is None and have):
        targets.append("ref")
        if shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc"):
            targets.append("gpu_optimised")  # the reference's GPU_Optimised decoder, sm_100a
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref_dir}", *targets], check=True)


class Oracle:
    """The C restatement (cmd_oracle.c), runtime-parameterised by set id."""

    def __init__(self, set_id: int):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(with_reference=False)
        self.lib = lib = ctypes.CDLL(path)
        lib.o_gf_mul.restype = ctypes.c_uint16
        lib.o_gf_inv.restype = ctypes.c_uint16
        lib.o_gf_frac.restype = ctypes.c_uint16
        lib.o_errorstream_format.restype = ctypes.c_long
        self.p = Params()
        if lib.o_params_get(int(set_id), ctypes.byref(self.p)) != 0:
            raise ValueError(f"unknown parameter set {set_id}")
        self.set_id = set_id
        self.m, self.n, self.t = self.p.m, self.p.n, self.p.t
        self.ct_bytes, self.sk_bytes, self.sb = self.p.ct_bytes, self.p.sk_bytes, self.p.sb
        self._key = None

    # -- field ------------------------------------------------------------
    def gf_mul(self, a: int, b: int) -> int:
        return self.lib.o_gf_mul(self.m, a, b)

    def gf_frac(self, den: int, num: int) -> int:
        return self.lib.o_gf_frac(self.m, den, num)

    def gf_mul_row(self, a: int) -> np.ndarray:
        out = np.zeros(1 << self.m, np.uint16)
        self.lib.o_gf_mul_row(self.m, a, _ptr(out, _u16p))
        return out

    def gf_frac_row(self, num: int) -> np.ndarray:
        out = np.zeros(1 << self.m, np.uint16)
        self.lib.o_gf_frac_row(self.m, num, _ptr(out, _u16p))
        return out

    # -- key --------------------------------------------------------------
    def support_from_cond(self, cond: bytes) -> np.ndarray:
        c = np.frombuffer(bytes(cond), np.uint8).copy()
        out = np.zeros(self.n, np.uint16)
        if self.lib.o_support_gen(ctypes.byref(self.p), _ptr(c, _u8p), _ptr(out, _u16p)):
            raise MemoryError
        return out

    def expand(self, sk: bytes):
        """Returns (g[t+1], L[n], inv_tab[sb, 2t])."""
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        g = np.zeros(self.t + 1, np.uint16)
        L = np.zeros(self.n, np.uint16)
        tab = np.zeros((self.sb, 2 * self.t), np.uint16)
        if self.lib.o_key_expand(ctypes.byref(self.p), _ptr(skb, _u8p), _ptr(g, _u16p),
                                 _ptr(L, _u16p), _ptr(tab, _u16p)):
            raise MemoryError
        self._key = (g, L, tab)
        return g, L, tab

    # -- stages -------------------------------------------------------------
    def synd(self, ct: bytes, tab: np.ndarray | None = None) -> np.ndarray:
        tab = self._key[2] if tab is None else tab
        c = np.frombuffer(bytes(ct), np.uint8).copy()
        s = np.zeros(2 * self.t, np.uint16)
        self.lib.o_synd(ctypes.byref(self.p), _ptr(np.ascontiguousarray(tab), _u16p),
                        _ptr(c, _u8p), _ptr(s, _u16p))
        return s

    def bm(self, s: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(s, np.uint16)
        loc = np.zeros(self.t + 1, np.uint16)
        self.lib.o_bm(ctypes.byref(self.p), _ptr(s, _u16p), _ptr(loc, _u16p))
        return loc

    def root(self, loc: np.ndarray, L: np.ndarray | None = None) -> np.ndarray:
        L = self._key[1] if L is None else L
        loc = np.ascontiguousarray(loc, np.uint16)
        L = np.ascontiguousarray(L, np.uint16)
        out = np.zeros(self.n, np.uint16)
        self.lib.o_root(ctypes.byref(self.p), _ptr(loc, _u16p), _ptr(L, _u16p), _ptr(out, _u16p))
        return out

    def decrypt(self, sk: bytes, cts: np.ndarray, nthreads: int = 1) -> np.ndarray:
        """cts: uint8 [count, ct_bytes] -> error bytes uint8 [count, n/8]."""
        cts = np.ascontiguousarray(cts, np.uint8).reshape(-1, self.ct_bytes)
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        err = np.zeros((cts.shape[0], self.n // 8), np.uint8)
        rc = self.lib.o_decrypt_batch(ctypes.byref(self.p), _ptr(skb, _u8p), _ptr(cts, _u8p),
                                      ctypes.c_size_t(cts.shape[0]), _ptr(err, _u8p), nthreads)
        if rc:
            raise RuntimeError("oracle decrypt failed")
        return err

    def decap(self, sk: bytes, cts: np.ndarray, nthreads: int = 1) -> tuple[np.ndarray, np.ndarray]:
        """Classic McEliece decapsulation around the reference's decrypt (no
        counterpart in the reference, which encapsulates only:
        kem/common/core/operations.c:15-34, K = SHAKE256(1 || e || C)).
        Returns (keys uint8 [count, 32], accept uint8 [count]): K =
        SHAKE256(b || v || C), b = accept, v = e or the sk's string s."""
        import hashlib
        cts = np.ascontiguousarray(cts, np.uint8).reshape(-1, self.ct_bytes)
        err = self.decrypt(sk, cts, nthreads)
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        acc = np.zeros(cts.shape[0], np.uint8)
        if self.lib.o_decap_accept(ctypes.byref(self.p), _ptr(skb, _u8p), _ptr(cts, _u8p), _ptr(err, _u8p),
                                   ctypes.c_size_t(cts.shape[0]), _ptr(acc, _u8p)):
            raise RuntimeError("oracle decap failed")
        s_off = 40 + 2 * self.t + (1 << (self.m - 4)) * (2 * self.m - 1)
        s = bytes(sk)[s_off: s_off + self.n // 8]
        keys = np.zeros((cts.shape[0], 32), np.uint8)
        for c in range(cts.shape[0]):
            pre = (b"\x01" + err[c].tobytes()) if acc[c] else (b"\x00" + s)
            keys[c] = np.frombuffer(hashlib.shake_256(pre + cts[c].tobytes()).digest(32), np.uint8)
        return keys, acc

    # -- key generation (crypto_kem_keypair, kem/common/core/operations.c:36-107)
    def kg_genpoly(self, f: np.ndarray):
        f = np.ascontiguousarray(f, np.uint16)
        irr = np.zeros(self.t, np.uint16)
        rc = self.lib.o_kg_genpoly(ctypes.byref(self.p), _ptr(f, _u16p), _ptr(irr, _u16p))
        return (irr if rc == 0 else None)

    def kg_pk_gen(self, irr: np.ndarray, perm: np.ndarray):
        irr = np.ascontiguousarray(irr, np.uint16)
        perm = np.ascontiguousarray(perm, np.uint32)
        mt = self.m * self.t
        pk = np.zeros(mt * ((self.n - mt + 7) // 8), np.uint8)
        pi = np.zeros(1 << self.m, np.int16)
        rc = self.lib.o_kg_pk_gen(ctypes.byref(self.p), _ptr(irr, _u16p), perm.ctypes.data_as(ctypes.c_void_p),
                                  _ptr(pk, _u8p), pi.ctypes.data_as(ctypes.c_void_p))
        return (pk, pi) if rc == 0 else None

    def kg_controlbits(self, pi: np.ndarray) -> np.ndarray:
        pi = np.ascontiguousarray(pi, np.int16)
        out = np.zeros(self.p.cond_bytes, np.uint8)
        self.lib.o_kg_controlbits(self.m, pi.ctypes.data_as(ctypes.c_void_p), _ptr(out, _u8p))
        return out

    def keypair(self, seed: bytes, max_attempts: int = 256):
        """Returns (pk bytes, sk bytes, attempts) of crypto_kem_keypair with
        randombytes() yielding `seed`; see keypair_from_seed."""
        return keypair_from_seed(self, seed, max_attempts)

    def encrypt(self, pk: bytes, errs: np.ndarray) -> np.ndarray:
        """Ciphertexts [count, ct_bytes] of error vectors [count, n/8] under a
        public key (kem/common/core/encrypt.c:87-120's syndrome rule)."""
        errs = np.ascontiguousarray(errs, np.uint8).reshape(-1, self.n // 8)
        pkb = np.frombuffer(bytes(pk), np.uint8).copy()
        out = np.zeros((errs.shape[0], self.ct_bytes), np.uint8)
        if self.lib.o_encrypt_batch(ctypes.byref(self.p), _ptr(pkb, _u8p), _ptr(errs, _u8p),
                                    ctypes.c_size_t(errs.shape[0]), _ptr(out, _u8p)):
            raise MemoryError
        return out

    def random_errors(self, seed: int, count: int) -> np.ndarray:
        """`count` error vectors [count, n/8] of weight exactly t, uniform
        over [0, n), from a seeded stream."""
        out = np.zeros((count, self.n // 8), np.uint8)
        self.lib.o_random_errors(ctypes.byref(self.p), ctypes.c_uint64(seed & (2 ** 64 - 1)),
                                 ctypes.c_size_t(count), _ptr(out, _u8p))
        return out

    def errorstream(self, err: np.ndarray) -> bytes:
        err = np.ascontiguousarray(err, np.uint8).reshape(-1, self.n // 8)
        cap = err.shape[0] * (1 + 6 * self.n // 8 * 8) + 16
        buf = ctypes.create_string_buffer(cap)
        got = self.lib.o_errorstream_format(ctypes.byref(self.p), _ptr(err, _u8p),
                                            ctypes.c_size_t(err.shape[0]), buf, ctypes.c_size_t(cap))
        if got < 0:
            raise RuntimeError("errorstream buffer too small")
        return buf.raw[:got]


def keypair_from_seed(stages, seed: bytes, max_attempts: int = 256):
    """crypto_kem_keypair (kem/common/core/operations.c:36-107) with
    randombytes() yielding the 32-byte `seed`, over a stage provider (the
    restatement ``Oracle`` or the reference's own ``RefKeygen``).  Each attempt
    expands 0x40 || seed with SHAKE256 into r = s (n/8) | perm (4 * 2^m) |
    f (2t) | next seed (32); a rejected attempt continues with the next seed.
    sk = seed | 0xFFFFFFFF as 8 bytes | irr (2t) | control bits | s."""
    import hashlib
    m, n, t = stages.m, stages.n, stages.t
    q = 1 << m
    rlen = n // 8 + 4 * q + 2 * t + 32
    seed = bytes(seed)
    assert len(seed) == 32
    for attempt in range(1, max_attempts + 1):
        r = hashlib.shake_256(b"\x40" + seed).digest(rlen)
        f = np.frombuffer(r, "<u2", t, rlen - 32 - 2 * t) & (q - 1)
        irr = stages.kg_genpoly(f)
        if irr is not None:
            perm = np.frombuffer(r, "<u4", q, rlen - 32 - 2 * t - 4 * q)
            got = stages.kg_pk_gen(irr, perm)
            if got is not None:
                pk, pi = got
                cond = stages.kg_controlbits(pi)
                sk = seed + bytes.fromhex("ffffffff00000000") + irr.astype("<u2").tobytes() + cond.tobytes() + r[: n // 8]
                return pk.tobytes(), sk, attempt
        seed = r[rlen - 32:]
    raise RuntimeError("no key after max_attempts")


class RefKeygen:
    """The reference's own kem/ key generation for one set
    (oracle/_ref/libkeygen_<set>.so): genpoly_gen, pk_gen, controlbits."""

    def __init__(self, set_id: int):
        path = os.path.join(HERE, "_ref", f"libkeygen_{set_id}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        info = (ctypes.c_int * 6)()
        self.lib.ref_kg_info(info)
        self.m, self.n, self.t, self.pk_rows, self.pk_row_bytes, self.cond_bytes = list(info)
        self.set_id = set_id

    @staticmethod
    def available(set_id: int) -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", f"libkeygen_{set_id}.so"))

    def kg_genpoly(self, f: np.ndarray):
        f = np.ascontiguousarray(f, np.uint16)
        irr = np.zeros(self.t, np.uint16)
        rc = self.lib.ref_kg_genpoly(f.ctypes.data_as(ctypes.c_void_p), irr.ctypes.data_as(ctypes.c_void_p))
        return irr if rc == 0 else None

    def kg_pk_gen(self, irr: np.ndarray, perm: np.ndarray):
        irr_b = np.ascontiguousarray(irr, "<u2").tobytes()
        perm = np.ascontiguousarray(perm, np.uint32)
        pk = np.zeros(self.pk_rows * self.pk_row_bytes, np.uint8)
        pi = np.zeros(1 << self.m, np.int16)
        rc = self.lib.ref_kg_pk_gen(pk.ctypes.data_as(ctypes.c_void_p), ctypes.c_char_p(irr_b),
                                    perm.ctypes.data_as(ctypes.c_void_p), pi.ctypes.data_as(ctypes.c_void_p))
        return (pk, pi) if rc == 0 else None

    def kg_controlbits(self, pi: np.ndarray) -> np.ndarray:
        pi = np.ascontiguousarray(pi, np.int16)
        out = np.zeros(self.cond_bytes, np.uint8)
        self.lib.ref_kg_controlbits(out.ctypes.data_as(ctypes.c_void_p), pi.ctypes.data_as(ctypes.c_void_p))
        return out

    def keypair(self, seed: bytes, max_attempts: int = 256):
        return keypair_from_seed(self, seed, max_attempts)


def reference_decrypt_rows(keys: list[tuple[int, bytes]], key_idx: np.ndarray, cts: np.ndarray,
                           nthreads: int = 0, row_bytes: int = 1024) -> tuple[np.ndarray, str]:
    """Decodes a batch that mixes keys and parameter sets with the reference's
    own CPU decoder (RefLib; the restatement where the reference build is
    absent).  keys[k] = (set id, secret key); row r is ciphertext cts[r] (its
    first ct_bytes bytes) under keys[key_idx[r]].  Returns (error rows
    [rows, row_bytes], zero past each set's n/8 bytes; the checker's kind:
    "reference" or "port")."""
    nthreads = nthreads or (os.cpu_count() or 1)
    key_idx = np.asarray(key_idx)
    out = np.zeros((key_idx.size, row_bytes), np.uint8)
    decs: dict[int, object] = {}
    kinds = set()
    order = np.argsort(key_idx, kind="stable")
    bounds = np.searchsorted(key_idx[order], np.arange(len(keys) + 1))
    for k, (s, sk) in enumerate(keys):
        rows = order[bounds[k]: bounds[k + 1]]
        if rows.size == 0:
            continue
        if s not in decs:
            decs[s] = RefLib(s) if RefLib.available(s) else Oracle(s)
            kinds.add("reference" if isinstance(decs[s], RefLib) else "port")
        d = decs[s]
        ctb = d.ct_bytes if hasattr(d, "ct_bytes") else d.p.ct_bytes
        e = d.decrypt(sk, np.ascontiguousarray(cts[rows, :ctb]), nthreads=min(nthreads, rows.size))
        out[rows, : e.shape[1]] = e
    return out, ("reference" if kinds == {"reference"} else "port" if kinds == {"port"} else "mixed")


class RefLib:
    """The reference's own CPU/ decoder for one set (oracle/_ref/libref_<set>.so)."""

    def __init__(self, set_id: int):
        path = os.path.join(HERE, "_ref", f"libref_{set_id}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = lib = ctypes.CDLL(path)
        for name in ("ref_gf_mul", "ref_gf_frac", "ref_gf_inv", "ref_bitrev"):
            getattr(lib, name).restype = ctypes.c_uint16
        info = (ctypes.c_int * 6)()
        lib.ref_info(info)
        self.m, self.n, self.t, self.ct_bytes, self.sk_bytes, self.sb = list(info)
        self.set_id = set_id

    @staticmethod
    def available(set_id: int) -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", f"libref_{set_id}.so"))

    def load_sk(self, sk: bytes) -> None:
        skb = np.frombuffer(bytes(sk), np.uint8).copy()
        self.lib.ref_load_sk(_ptr(skb, _u8p))

    def support(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint16)
        self.lib.ref_get_support(_ptr(out, _u16p))
        return out

    def goppa(self) -> np.ndarray:
        out = np.zeros(self.t + 1, np.uint16)
        self.lib.ref_get_goppa(_ptr(out, _u16p))
        return out

    def inverse_table(self) -> np.ndarray:
        out = np.zeros((self.sb, 2 * self.t), np.uint16)
        self.lib.ref_get_inverse_table(_ptr(out, _u16p))
        return out

    def support_from_cond(self, cond: bytes) -> np.ndarray:
        c = np.frombuffer(bytes(cond), np.uint8).copy()
        out = np.zeros(self.n, np.uint16)
        self.lib.ref_support_from_cond(_ptr(c, _u8p), _ptr(out, _u16p))
        return out

    def synd(self, ct: bytes) -> np.ndarray:
        c = np.frombuffer(bytes(ct), np.uint8).copy()
        s = np.zeros(2 * self.t, np.uint16)
        self.lib.ref_synd(_ptr(c, _u8p), _ptr(s, _u16p))
        return s

    def bm(self, s: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(s, np.uint16)
        loc = np.zeros(self.t + 1, np.uint16)
        self.lib.ref_bm(_ptr(s, _u16p), _ptr(loc, _u16p))
        return loc

    def root(self, loc: np.ndarray) -> np.ndarray:
        loc = np.ascontiguousarray(loc, np.uint16)
        out = np.zeros(self.n, np.uint16)
        self.lib.ref_root(_ptr(loc, _u16p), _ptr(out, _u16p))
        return out

    def gf_mul_row(self, a: int) -> np.ndarray:
        out = np.zeros(1 << self.m, np.uint16)
        self.lib.ref_gf_mul_row(a, _ptr(out, _u16p))
        return out

    def gf_frac_row(self, num: int) -> np.ndarray:
        out = np.zeros(1 << self.m, np.uint16)
        self.lib.ref_gf_frac_row(num, _ptr(out, _u16p))
        return out

    def decrypt(self, sk: bytes, cts: np.ndarray, nthreads: int = 1) -> np.ndarray:
        self.load_sk(sk)
        cts = np.ascontiguousarray(cts, np.uint8).reshape(-1, self.ct_bytes)
        err = np.zeros((cts.shape[0], self.n // 8), np.uint8)
        if self.lib.ref_decrypt_batch(_ptr(cts, _u8p), ctypes.c_size_t(cts.shape[0]),
                                      _ptr(err, _u8p), nthreads):
            raise RuntimeError("reference decrypt failed")
        return err
