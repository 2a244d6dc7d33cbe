"""sgmas_morton_codes_noalloc: Morton codes for callers that cannot allocate
device memory (hosts that hand out device memory from their own pool or fix
it at start-up, loops that must not allocate once they run).  The entry point keeps its reduction
scratch in a fixed static device array, so it must give exactly the codes of
the allocating entry point sgmas_morton_codes -- on consecutive calls that
share that array -- and refuse inputs larger than the array can serve.

This file sorts last so that a run stopping at its first failure has run
every other test first; it also passes on its own in a fresh process."""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SGMAS_ERR_CAPACITY = -4


def _positions(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.3, 0.7, size=(n, 3))
    pos[::7] = pos[0]            # repeated points share codes (ties broken by index)
    return torch.from_numpy(pos).cuda()


def _reference_codes(sgmas, pos):
    ctx = sgmas.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    out = torch.zeros(pos.shape[0], dtype=torch.int64, device="cuda")
    ctx.morton_codes(pos, out)
    torch.cuda.synchronize()
    ctx.close()
    return out.cpu().numpy().view(np.uint64)


def test_noalloc_matches_allocating_entry_on_consecutive_calls():
    import sgmas
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row on different inputs: the shared static scratch keeps the
    # first call's partial boxes, which must not leak into the second result
    for n, seed in ((100_003, 1), (4_097, 2)):
        pos = _positions(n, seed)
        codes = torch.zeros(n, dtype=torch.int64, device="cuda")
        assert sgmas.morton_codes_noalloc(pos, codes, stream=stream) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(codes.cpu().numpy().view(np.uint64), _reference_codes(sgmas, pos))


def test_noalloc_with_given_box_and_size_limit():
    import sgmas
    stream = torch.cuda.current_stream().cuda_stream
    pos = _positions(20_000, 3)
    box = np.array([-0.5, -0.5, -0.5, 1.0, 1.0, 1.0])
    codes = torch.zeros(20_000, dtype=torch.int64, device="cuda")
    assert sgmas.morton_codes_noalloc(pos, codes, aabb=box, stream=stream) == 0
    ctx = sgmas.Context(0)
    ctx.set_stream(stream)
    ref = torch.zeros_like(codes)
    ctx.morton_codes(pos, ref, aabb=box)
    torch.cuda.synchronize()
    ctx.close()
    np.testing.assert_array_equal(codes.cpu().numpy(), ref.cpu().numpy())
    # one vertex more than the static scratch serves: refused before any work is queued
    too_many = sgmas.MORTON_NOALLOC_MAX_VERTS + 1
    assert sgmas.morton_codes_noalloc(pos, codes, stream=stream, n=too_many) == SGMAS_ERR_CAPACITY
