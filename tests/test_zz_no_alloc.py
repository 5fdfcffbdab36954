"""GPU: psg_count_noalloc(), the entry point for callers that cannot
allocate device memory while they count (an allocator's own callbacks,
real-time loops where a cudaMalloc could synchronise the device, embedders
with a fixed memory budget). It keeps all
of its scratch in one fixed static device array, so these tests check that
back-to-back calls (which reuse that array) give exactly what psg_count()
gives, and that a stop beyond its limit is refused with a clear error.

Named test_zz_* so that pytest collects it last; it also passes alone in a
fresh process."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 36


def noalloc(psg, start, stop, kinds, out, stream):
    return psg.load().psg_count_noalloc(start, stop, kinds, ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_matches_psg_count_twice(psg):
    import torch
    stream = torch.cuda.Stream()
    with psg.Context(device=torch.cuda.current_device()) as ctx:
        out = torch.full((6,), -1, dtype=torch.int64, device="cuda")
        # two calls in a row share the static scratch: the second must not
        # see the first one's counts
        for a, b, k in [(0, 10 ** 9, 0x3F), (10 ** 10, 10 ** 10 + 10 ** 8, 0x3F),
                        (LIMIT - 10 ** 7, LIMIT, 0x3F), (0, 30, 0x3F), (3, 100, 0x5)]:
            with torch.cuda.stream(stream):
                assert noalloc(psg, a, b, k, out, stream) == 0, psg.load().psg_last_error()
            stream.synchronize()
            got = [int(x) for x in out.tolist()]
            assert got == ctx.count(a, b, k), (a, b, k, got)


def test_noalloc_rejects_stop_beyond_limit(psg):
    import torch
    out = torch.zeros(6, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = noalloc(psg, LIMIT - 100, LIMIT + 1, 0x3F, out, stream)
    assert rc == 5                                           # PSG_ERR_LIMIT
    assert b"2^36" in psg.load().psg_last_error()
    assert noalloc(psg, 0, 100, 1, out, stream) == 0         # still usable afterwards
    torch.cuda.synchronize()
    assert out.tolist() == [25, 0, 0, 0, 0, 0]
