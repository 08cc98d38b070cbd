"""The allocation-free photon grid entry point (srt_photon_grid_build_noalloc).

Callers that cannot call cudaMalloc — an engine or framework whose pool
allocator owns the GPU's memory, or a frame loop that forbids allocation
while it runs — use this entry point: it works only on device buffers the
caller owns and takes its temporary storage from a fixed array inside the
library.  This test (the caller here allocates its buffers with torch) checks,
through the C ABI and on calls in a row that share that array:

* the keys and ranges equal the CPU oracle's (build_grid.wgsl:25-73, sort
  form) and the allocating entry point srt_photon_grid_build's, bit for bit
  (integer results), at 22 and 20 hash bits;
* n = 0 only clears the ranges, and either output may be NULL;
* an oversized request is refused.

Misaligned pointers are refused before any device work; that is checked on
the CPU (tests/test_abi_host.py), never by handing a GPU a bad address.

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


def _call(L, stream, d_ph, n, frame, bits, d_keys, d_ranges):
    return L.srt_photon_grid_build_noalloc(C.c_void_p(stream), C.c_void_p(d_ph.data_ptr()) if d_ph is not None else None,
                                           n, frame, 0.02, bits,
                                           C.c_void_p(d_keys.data_ptr()) if d_keys is not None else None,
                                           C.c_void_p(d_ranges.data_ptr()) if d_ranges is not None else None)


def test_noalloc_grid_matches_oracle_and_allocating_entry_point(srt, orc):
    torch = pytest.importorskip("torch")
    L = srt.lib()
    ctx = srt.Context(0)
    stream = torch.cuda.current_stream().cuda_stream
    # calls in a row; later ones are smaller, so stale scratch would show
    for n, frame, spread, bits in ((1 << 20, 7, 0.5, 22), (50_000, 8, 0.2, 22), (200_003, 9, 0.3, 20)):
        ph = _photons(n, n + frame, spread)
        d_ph = torch.from_numpy(ph).cuda()
        d_keys = torch.zeros(n, dtype=torch.int64, device="cuda")
        d_ranges = torch.full((1 << bits, 2), 0x7FFFFFFF, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        st = _call(L, stream, d_ph, n, frame, bits, d_keys, d_ranges)
        assert st == 0, srt.STATUS.get(st, st)
        torch.cuda.synchronize()
        keys = d_keys.cpu().numpy().view(np.uint64)
        ranges = d_ranges.cpu().numpy().view(np.uint32)
        o_keys, o_ranges = orc.photon_grid_build(ph, frame, 0.02, bits)
        assert np.array_equal(keys, o_keys)
        assert np.array_equal(ranges, o_ranges.reshape(ranges.shape))
        ref_keys, ref_ranges = srt.photon_grid_build(ctx, ph, frame, 0.02, bits)
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(ranges, ref_ranges)

        # keys only: ranges untouched; ranges only: the same ranges
        d_keys2 = torch.zeros(n, dtype=torch.int64, device="cuda")
        st = _call(L, stream, d_ph, n, frame, bits, d_keys2, None)
        assert st == 0
        d_ranges2 = torch.full((1 << bits, 2), 0x7FFFFFFF, dtype=torch.int32, device="cuda")
        st = _call(L, stream, d_ph, n, frame, bits, None, d_ranges2)
        assert st == 0
        torch.cuda.synchronize()
        assert np.array_equal(d_keys2.cpu().numpy().view(np.uint64), o_keys)
        assert np.array_equal(d_ranges2.cpu().numpy().view(np.uint32), ranges)

    # n = 0: the ranges are cleared and nothing else happens
    d_ranges = torch.full((1 << 20, 2), 0x7FFFFFFF, dtype=torch.int32, device="cuda")
    st = _call(L, stream, None, 0, 3, 20, None, d_ranges)
    assert st == 0
    torch.cuda.synchronize()
    assert int(d_ranges.abs().sum().item()) == 0

    # a request above the fixed capacity is refused before any device work
    st = L.srt_photon_grid_build_noalloc(C.c_void_p(stream), C.c_void_p(256), (1 << 20) + 1, 0, 0.02, 22, None, None)
    assert srt.STATUS[st] == "CAPACITY"
    ctx.close()
