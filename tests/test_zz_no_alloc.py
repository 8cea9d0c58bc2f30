"""fcb_conservation_sum_noalloc: the mass sums of fcb_conservation_check, for
callers that cannot allocate device memory while they run (a serving loop whose
HBM is committed to admitted solves, code that must not let cudaMalloc/cudaFree
synchronise the device, hosts that own all device memory).  The entry point
works out of a fixed array inside the library; this file checks, through the
C ABI, that two calls in a row give the context's own sums and that the calls
leave the device's free memory unchanged.  It runs last so that a failure here
leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

REL_TOL = 1e-13  # the tolerance of the mass tests in test_gpu_parity.py
SCRATCH_BYTES = 262144 * 8  # the fixed array inside the library


def _device_inputs(solver, torch):
    o = solver.options
    q = torch.from_numpy(solver.get_q()).to("cuda")  # (patches, meqn, ny, nx), contiguous
    areas = []
    for p in range(solver.num_patches):
        level, _, _ = solver.patch_info(p)
        dx = 1.0 / (2 ** level) / o.mx
        dy = 1.0 / (2 ** level) / o.my
        areas.append(dx * dy)
    area = torch.tensor(areas, dtype=torch.float64, device="cuda")
    return q, area


def _call(lib, q, area, out, o, stream):
    psize = o.meqn * o.ny * o.nx
    return lib.fcb_conservation_sum_noalloc(
        ctypes.c_void_p(q.data_ptr()), ctypes.c_size_t(psize), q.shape[0], o.mx, o.my, o.mbc, o.meqn,
        ctypes.c_void_p(area.data_ptr()), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_mass_matches_context_on_two_calls(gpu_lib):
    import torch

    import forestclaw_b200 as fcb

    lib = fcb.lib()
    cfg = cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=16)
    s = fcb.Solver(cases.to_options(cfg))
    s.initialize()
    o = s.options
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.empty(o.meqn, dtype=torch.float64, device="cuda")

    for call, t in enumerate((0.0, 0.005)):
        s.advance_all_levels(t, 0.005)   # a different state for each call
        want = s.conservation_check()    # the existing entry point
        q, area = _device_inputs(s, torch)
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rc = _call(lib, q, area, out, o, stream)
        assert rc == 0, lib.fcb_last_error().decode()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=REL_TOL, atol=0.0, err_msg=f"call {call}")
        # The first use of the library's module on a device may materialise the
        # fixed array (CUDA loads modules lazily); after that no call takes memory.
        limit = SCRATCH_BYTES if call == 0 else 0
        assert 0 <= free0 - free1 <= limit, f"call {call} changed device free memory by {free0 - free1} bytes"
    s.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch(gpu_lib):
    import torch

    import forestclaw_b200 as fcb

    lib = fcb.lib()
    q = torch.zeros(1, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    # 70,000 patches x 4 components = 280,000 > 262,144 per-patch sums
    rc = lib.fcb_conservation_sum_noalloc(
        ctypes.c_void_p(q.data_ptr()), ctypes.c_size_t(4 * 12 * 12), 70000, 8, 8, 2, 4,
        ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1  # FCB_ERR_INVALID, nothing launched
    assert b"exceeds the fixed scratch" in lib.fcb_last_error()
