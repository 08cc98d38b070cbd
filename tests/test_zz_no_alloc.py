"""The allocation-free photon grid entry point (srt_photon_grid_build_noalloc).

Callers that cannot call cudaMalloc — an engine or framework whose pool
allocator owns the GPU's memory, or a frame loop that forbids allocation
while it runs — use this entry point: it works only on device buffers the
caller owns and takes its temporary storage from a fixed array inside the
library.  This test (the caller here allocates its buffers with torch) checks
that two calls in a row, through the C ABI, give exactly the keys and ranges
of the allocating entry point srt_photon_grid_build (integer results:
bit-exact), and that an oversized request is refused.

Kept in its own file, collected last, so that a failure here comes after
every other test has run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _photons(n, seed, spread):
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 8), np.float32)
    p[:, 0:3] = rng.uniform(-spread, spread, (n, 3))
    p[: n // 10, 0:3] = p[0, 0:3]  # one crowded cell
    p[:, 3] = rng.uniform(380, 780, n)
    p[:, 4:7] = rng.normal(size=(n, 3))
    p[:, 7] = rng.uniform(0.01, 4, n)
    p[rng.integers(0, n, max(1, n // 40)), 7] = 0.0
    return p


def test_noalloc_grid_matches_allocating_entry_point(srt):
    torch = pytest.importorskip("torch")
    L = srt.lib()
    ctx = srt.Context(0)
    bits = 22
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row; the second is smaller so stale scratch would show
    for n, frame, spread in ((1 << 20, 7, 0.5), (50_000, 8, 0.2)):
        ph = _photons(n, n + frame, spread)
        d_ph = torch.from_numpy(ph).cuda()
        d_keys = torch.zeros(n, dtype=torch.int64, device="cuda")
        d_ranges = torch.full((1 << bits, 2), 0x7FFFFFFF, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        st = L.srt_photon_grid_build_noalloc(C.c_void_p(stream), C.c_void_p(d_ph.data_ptr()), n, frame, 0.02, bits,
                                             C.c_void_p(d_keys.data_ptr()), C.c_void_p(d_ranges.data_ptr()))
        assert st == 0, srt.STATUS.get(st, st)
        torch.cuda.synchronize()
        keys = d_keys.cpu().numpy().view(np.uint64)
        ranges = d_ranges.cpu().numpy().view(np.uint32)
        ref_keys, ref_ranges = srt.photon_grid_build(ctx, ph, frame, 0.02, bits)
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(ranges, ref_ranges)
    # a request above the fixed capacity is refused before any device work
    st = L.srt_photon_grid_build_noalloc(C.c_void_p(stream), C.c_void_p(1), (1 << 20) + 1, 0, 0.02, bits, None, None)
    assert srt.STATUS[st] == "CAPACITY"
    ctx.close()
