"""The allocation-free fit entry point (PTB_FittingDeviceNoAlloc) against the regular Fitting export.

PTB_FittingDeviceNoAlloc serves callers that cannot allocate device memory themselves (for example code running
inside another runtime's stream callbacks, or under a fixed pre-sized memory pool): they pass device buffers for the
stack, the positions and the output, and the library works in a static device array instead of allocating. This file
is collected last so that a failure here never hides the other tests; it passes alone and after them.
"""
import numpy as np
import pytest

from conftest import GAUSS_PARAMS

pytestmark = pytest.mark.gpu


def _positions(rows):
    return np.ascontiguousarray(np.stack([rows[:, 0], rows[:, 1], rows[:, 4], rows[:, 5], rows[:, 15], rows[:, 16]], axis=1))


def _call_noalloc(lib, torch, stack, pos, fit, params):
    d_stack = torch.from_numpy(np.ascontiguousarray(stack).view(np.int16)).cuda()
    d_pos = torch.from_numpy(pos).cuda()
    d_out = torch.full((pos.shape[0] * 18,), -7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    n = lib.fitting_device_noalloc(d_stack.data_ptr(), d_pos.data_ptr(), pos.shape[0], d_out.data_ptr(), stack.shape, fit, params,
                                   stream.cuda_stream)
    torch.cuda.synchronize()
    assert n == pos.shape[0] * 18, lib.last_error()
    return d_out.cpu().numpy().reshape(-1, 18)


def test_no_alloc_fitting_matches_fitting_on_two_calls(lib, orc, stacks):
    import torch
    st = stacks["stack"]
    det = orc.localization(st, 103.6, 0.0, 0, GAUSS_PARAMS)
    pos_a = _positions(det)
    pos_b = _positions(det[::3])
    pos_b[5, 1] = st.shape[0] + 4  # a plane outside the stack: border sentinel row, like Fitting
    # two calls in a row on the same static scratch: different sizes and modes; the second must not see the first
    for pos, fit in ((pos_a, 2), (pos_b, 4)):
        expected = lib.fitting(st, pos, fit, GAUSS_PARAMS)
        got = _call_noalloc(lib, torch, st, pos, fit, GAUSS_PARAMS)
        assert got.shape == expected.shape
        # same kernels on the same inputs: identical within the tests' tolerance (in practice bit for bit)
        assert np.allclose(got, expected, rtol=1e-12, atol=1e-12, equal_nan=True)
        assert np.array_equal(got[:, 2], expected[:, 2])  # per-plane Index column


def test_no_alloc_rejects_oversized_calls(lib, stacks):
    import torch
    st = stacks["stack"][:1]
    n = 65537
    pos = np.zeros((n, 6))
    pos[:, 1] = 1
    d_stack = torch.from_numpy(np.ascontiguousarray(st).view(np.int16)).cuda()
    d_pos = torch.from_numpy(pos).cuda()
    d_out = torch.zeros(n * 18, dtype=torch.float64, device="cuda")
    got = lib.fitting_device_noalloc(d_stack.data_ptr(), d_pos.data_ptr(), n, d_out.data_ptr(), st.shape, 2, GAUSS_PARAMS)
    assert got == 0 and "65536" in lib.last_error()
