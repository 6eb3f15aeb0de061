"""The allocation-free compaction entry point (lk_compact_ge_noalloc).

Some callers cannot allocate device memory where they compact: a host
framework that owns all device memory through its own pool and forbids direct
cudaMalloc calls, or a latency-critical loop where an allocation (which may
synchronise the device) is not allowed. lk_compact_ge_noalloc keeps its
scratch in a static device array inside the library instead. This test calls
it through the C ABI twice in a row (the second call smaller, so stale
contents of the shared array would show) and checks every output against the
allocating entry point lk_compact_ge, exactly (indices are integers; values
are copies of the inputs). It also checks that sizes beyond the array's limit
are rejected. The file is named so that pytest collects it last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compact_both(lib, torch, scores, thr, cap):
    from loki_b200 import _capi as C

    n = scores.numel()
    stream = torch.cuda.current_stream().cuda_stream
    out = {}
    # Existing entry point: caller-provided scratch.
    scratch = torch.empty(int(lib.lk_compact_scratch_bytes(n)), dtype=torch.uint8, device="cuda")
    idx = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
    val = torch.full((cap,), np.nan, dtype=torch.float32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    C.check(lib.lk_compact_ge(scores.data_ptr(), n, thr, idx.data_ptr(), val.data_ptr(), cap,
                              cnt.data_ptr(), scratch.data_ptr(), stream))
    out["alloc"] = (idx, val, cnt)
    # Allocation-free entry point: no scratch argument.
    idx2 = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
    val2 = torch.full((cap,), np.nan, dtype=torch.float32, device="cuda")
    cnt2 = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    C.check(lib.lk_compact_ge_noalloc(scores.data_ptr(), n, thr, idx2.data_ptr(), val2.data_ptr(), cap,
                                      cnt2.data_ptr(), stream))
    out["noalloc"] = (idx2, val2, cnt2)
    torch.cuda.synchronize()
    return out


def test_noalloc_compaction_matches_allocating_entry_point(cuda):
    from loki_b200 import _capi as C

    torch = cuda
    lib = C.lib()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    # Two calls in a row: a large one, then a smaller one over fewer tiles.
    for n, thr, cap in [(5_000_003, 1.0, 1 << 21), (70_001, 0.5, 1 << 15)]:
        scores = torch.randn(n, generator=gen, device="cuda", dtype=torch.float32)
        scores[::97] = thr  # ties at the threshold are kept (>=)
        res = _compact_both(lib, torch, scores, thr, cap)
        i1, v1, c1 = res["alloc"]
        i2, v2, c2 = res["noalloc"]
        total = int(c1.item())
        assert total > 0 and total == int(c2.item())
        k = min(total, cap)
        assert torch.equal(i1[:k], i2[:k])
        assert torch.equal(v1[:k].view(torch.int32), v2[:k].view(torch.int32))
        # and both are the ordered >= selection
        want = torch.nonzero(scores >= thr).flatten()[:k].to(torch.int32)
        assert torch.equal(i2[:k], want)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    from loki_b200 import _capi as C

    torch = cuda
    lib = C.lib()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    # The size check happens before any launch, so no memory beyond `buf` is touched.
    rc = lib.lk_compact_ge_noalloc(buf.data_ptr(), (1 << 28) + 1, 0.0, None, None, 0, cnt.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    assert rc == C.LK_ERR_INVALID_ARG
    assert "2^28" in lib.lk_last_error().decode()
