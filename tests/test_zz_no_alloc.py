"""The allocation-free Sellp slice-set entry point.

It exists for callers that cannot allocate device memory (a host that owns
all device memory as one fixed arena, or a loop that must not call cudaMalloc
because it can synchronise the device): its scan scratch is a static array
inside the library.  Checked here through the C ABI against the workspace
entry point on two calls in a row, with different inputs, so stale scratch
contents from the first call would show up in the second.  This file is
collected last (pytest orders files by name).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from ginkgo_b200 import _lib, stencils

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _with_workspace(rp, slice_size, stride_factor):
    n = rp.numel() - 1
    ns = (n + slice_size - 1) // slice_size
    sets = torch.empty(ns + 1, dtype=torch.int64, device="cuda")
    lens = torch.empty(max(ns, 1), dtype=torch.int64, device="cuda")
    wsb = _lib.lib().b2s_sellp_slice_sets_workspace_bytes(n, slice_size)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("b2s_sellp_compute_slice_sets", n, _p(rp), slice_size,
              stride_factor, _p(sets), _p(lens), _p(ws), wsb, stream)
    return sets, lens[:ns]


def _no_alloc(rp, slice_size, stride_factor):
    n = rp.numel() - 1
    ns = (n + slice_size - 1) // slice_size
    sets = torch.full((ns + 1,), -7, dtype=torch.int64, device="cuda")
    lens = torch.full((max(ns, 1),), -7, dtype=torch.int64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("b2s_sellp_compute_slice_sets_noalloc", n, _p(rp), slice_size,
              stride_factor, _p(sets), _p(lens), stream)
    return sets, lens[:ns]


def test_no_alloc_slice_sets_match_workspace_entry_point_twice():
    cases = [
        # several scan tiles, long uneven rows
        (stencils.power_law(300000, seed=8, mu=2.0, max_len=900)[0], 32, 1),
        # a smaller matrix second: any leftover scratch would corrupt it
        (stencils.poisson_3d_7pt(20)[0], 7, 3),
    ]
    for rp_np, ss, sf in cases:
        rp = torch.from_numpy(rp_np).cuda()
        ref_sets, ref_lens = _with_workspace(rp, ss, sf)
        got_sets, got_lens = _no_alloc(rp, ss, sf)
        torch.cuda.synchronize()
        assert torch.equal(got_sets, ref_sets)
        assert torch.equal(got_lens, ref_lens)
        # and against the host restatement of compute_slice_sets
        n = len(rp_np) - 1
        lens_h = np.diff(rp_np).reshape(-1)
        pad = (-n) % ss
        lens_h = np.concatenate([lens_h, np.zeros(pad, lens_h.dtype)])
        exp_lens = ((lens_h.reshape(-1, ss) + sf - 1) // sf * sf).max(axis=1)
        assert np.array_equal(got_lens.cpu().numpy(), exp_lens)
        assert np.array_equal(got_sets.cpu().numpy(),
                              np.concatenate([[0], np.cumsum(exp_lens)]))


def test_no_alloc_rejects_more_slices_than_its_scratch():
    lib = _lib.lib()
    fake = C.c_void_p(16)  # rejected before any device access
    rc = lib.b2s_sellp_compute_slice_sets_noalloc(
        (4095 * 2048 + 1) * 32, fake, 32, 1, fake, fake, None)
    assert rc == -1
    assert b"static scratch" in lib.b2s_last_error()
