"""The allocation-free entry point, cmd_decrypt_plain_noalloc, for callers that
must not have the library allocate device memory (a framework-owned memory
pool, or a latency-critical loop that cannot take a cudaMalloc).

Called through the C ABI, twice in a row, on different batches: each call's
error vectors and weights must equal, bit for bit, those of the allocating
entry point cmd_decrypt_device on the same plain kernel path.  The first call
on a fresh engine must leave the engine's device-memory use and the device's
free memory unchanged; the second runs on a caller's stream without a weight
output.  A batch above CMD_NOALLOC_MAX_CTS is refused with CMD_E_ARG.  Named
so pytest collects it last; it also passes alone in a fresh process.
"""
from __future__ import annotations

import pytest
import torch

import cm_decrypt__b200 as cmd
from conftest import golden_sk

pytestmark = pytest.mark.gpu

NOALLOC_MAX = 4096  # CMD_NOALLOC_MAX_CTS in include/cmd_b200.h


def _outputs(n: int, info: cmd.SetInfo):
    return (torch.zeros((n, info.err_words), dtype=torch.int32, device="cuda"),
            torch.zeros(n, dtype=torch.int16, device="cuda"))


@pytest.mark.parametrize("set_id", [6960119, 348864])
def test_noalloc_matches_allocating_entry_point(set_id):
    L = cmd.lib()
    with cmd.Engine(0) as eng:
        key = cmd.Key(eng, set_id, golden_sk(set_id))
        info = key.info
        pk = cmd.PubKey(set_id, golden_sk(set_id))
        try:
            batches = []
            for count, seed in [(NOALLOC_MAX, 1), (1537, 2)]:
                cts, _, _ = pk.ciphertexts(seed=seed, count=count, malformed_permille=150)
                got_err, got_w = _outputs(count, info)
                got_err.fill_(-1)  # the no-alloc call must write every word
                batches.append((count, torch.from_numpy(cts).cuda(), got_err, got_w))
            stream = torch.cuda.Stream()
            torch.cuda.synchronize()

            # call 1: the first no-alloc call on this engine allocates nothing
            count, d_ct, got_err, got_w = batches[0]
            used0 = eng.memory()[0]
            free0 = torch.cuda.mem_get_info()[0]
            rc = L.cmd_decrypt_plain_noalloc(key.handle, d_ct.data_ptr(), count, got_err.data_ptr(),
                                             got_w.data_ptr(), None)
            assert rc == cmd.CMD_OK, cmd._last_error()
            torch.cuda.synchronize()
            assert eng.memory()[0] == used0, "the no-alloc call grew the engine's device memory"
            assert torch.cuda.mem_get_info()[0] == free0, "the no-alloc call allocated device memory"

            # call 2: a caller's stream, no weight output
            count2, d_ct2, got_err2, _ = batches[1]
            rc = L.cmd_decrypt_plain_noalloc(key.handle, d_ct2.data_ptr(), count2, got_err2.data_ptr(), None,
                                             stream.cuda_stream)
            assert rc == cmd.CMD_OK, cmd._last_error()
            stream.synchronize()

            for call, (n, d, e, w) in enumerate(batches):
                ref_err, ref_w = _outputs(n, info)
                rc = L.cmd_decrypt_device(eng.handle, key.handle, cmd.PATHS["plain"], d.data_ptr(), n,
                                          ref_err.data_ptr(), ref_w.data_ptr(), None)
                assert rc == cmd.CMD_OK
                torch.cuda.synchronize()
                assert torch.equal(e, ref_err), f"call {call}: error vectors differ"
                if call == 0:
                    assert torch.equal(w, ref_w), "call 0: weights differ"
                else:
                    assert not w.any(), "call 1 had no weight output and must not write one"

            d_ct = torch.zeros((NOALLOC_MAX + 1) * info.ct_bytes, dtype=torch.uint8, device="cuda")
            e, w = _outputs(NOALLOC_MAX + 1, info)
            rc = L.cmd_decrypt_plain_noalloc(key.handle, d_ct.data_ptr(), NOALLOC_MAX + 1, e.data_ptr(),
                                             w.data_ptr(), None)
            assert rc == cmd.CMD_E_ARG
            assert "maximum" in cmd._last_error()
        finally:
            key.free()

