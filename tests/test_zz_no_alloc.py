"""fcb_conservation_sum_noalloc: the mass sums of fcb_conservation_check, for
callers that cannot allocate device memory while they run (a serving loop whose
HBM is committed to admitted solves, code that must not let cudaMalloc/cudaFree
synchronise the device, hosts that own all device memory).  The entry point
works out of a fixed array inside the library; this file checks, through the
C ABI, that two calls in a row give the context's own sums and that the calls
leave the device's free memory unchanged, and, against a NumPy restatement of
the same Kahan sums, a padded patch stride and a call at exactly the size
limit.  It runs last so that a failure here leaves every other test already
run.
"""
import ctypes

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

MAX_SUMS = 262144  # per-patch sums the library's fixed array holds
SCRATCH_BYTES = MAX_SUMS * 8
ROOT = 1 << 28  # patch corners come in units of 2^-28 of the block


def _patch_area(o, level, x, y):
    """dx*dy of a leaf as the library computes it: the physical corners
    ax + (bx-ax)*x of the block coordinates, (xupper - xlower)/mx."""
    ax, bx, ay, by = o.extent
    h = ROOT >> level
    xl, xu = x / ROOT, (x + h) / ROOT
    yl, yu = y / ROOT, (y + h) / ROOT
    dx = ((ax + (bx - ax) * xu) - (ax + (bx - ax) * xl)) / o.mx
    dy = ((ay + (by - ay) * yu) - (ay + (by - ay) * yl)) / o.my
    return dx * dy


def _device_inputs(solver, torch):
    o = solver.options
    q = torch.from_numpy(solver.get_q()).to("cuda")  # (patches, meqn, ny, nx), contiguous
    areas = [_patch_area(o, *solver.patch_info(p)) for p in range(solver.num_patches)]
    area = torch.tensor(areas, dtype=torch.float64, device="cuda")
    return q, area


def _call(lib, q, area, out, npatches, stride, mx, my, mbc, meqn, stream):
    return lib.fcb_conservation_sum_noalloc(
        ctypes.c_void_p(q.data_ptr()), ctypes.c_size_t(stride), npatches, mx, my, mbc, meqn,
        ctypes.c_void_p(area.data_ptr()), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def _kahan_reference(q, area, mx, my, mbc):
    """NumPy restatement: Kahan over each patch's interior (component, then j,
    then i; fclaw2d_clawpatch46_diagnostics.f:13-58), then Kahan over the
    patches in order.  q is (patches, meqn, ny, nx)."""
    npatches, meqn = q.shape[:2]
    s = np.zeros((npatches, meqn))
    c = np.zeros((npatches, meqn))
    for j in range(mbc, mbc + my):
        for i in range(mbc, mbc + mx):
            y = q[:, :, j, i] * area[:, None] - c
            t = s + y
            c = (t - s) - y
            s = t
    total = []
    for m in range(meqn):
        acc, comp = 0.0, 0.0
        for v in s[:, m].tolist():
            y = v - comp
            t = acc + y
            comp = (t - acc) - y
            acc = t
        total.append(acc)
    return np.array(total)


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
        rc = _call(lib, q, area, out, q.shape[0], o.meqn * o.ny * o.nx, o.mx, o.my, o.mbc, o.meqn, stream)
        assert rc == 0, lib.fcb_last_error().decode()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        got = out.cpu().numpy()
        # the same Kahan sums in the same order, both built without FMA contraction
        assert np.array_equal(got, want), f"call {call}: {got} vs {want}"
        # The first use of the library's module on a device may materialise the
        # fixed array (CUDA loads modules lazily); after that no call takes memory.
        limit = SCRATCH_BYTES if call == 0 else 0
        assert 0 <= free0 - free1 <= limit, f"call {call} changed device free memory by {free0 - free1} bytes"
    s.close()


def test_noalloc_padded_stride_and_size_limit(gpu_lib):
    """A patch stride with 17 doubles of padding between patches, and a call
    with npatches * meqn exactly at the limit (262,144 patches of 4 x 4 cells):
    both equal the NumPy Kahan sums bit for bit."""
    import torch

    import forestclaw_b200 as fcb

    lib = fcb.lib()
    rng = np.random.default_rng(7)
    stream = torch.cuda.current_stream().cuda_stream
    for npatches, mx, meqn, pad in ((37, 8, 3, 17), (MAX_SUMS, 4, 1, 0)):
        mbc = 2
        n = mx + 2 * mbc
        psize = meqn * n * n
        qh = rng.uniform(0.5, 2.0, size=(npatches, psize + pad))
        ah = rng.uniform(1e-4, 1e-3, size=npatches)
        want = _kahan_reference(qh[:, :psize].reshape(npatches, meqn, n, n), ah, mx, mx, mbc)
        q = torch.from_numpy(qh).to("cuda")
        area = torch.from_numpy(ah).to("cuda")
        out = torch.full((meqn,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):
            rc = _call(lib, q, area, out, npatches, psize + pad, mx, mx, mbc, meqn, stream)
            assert rc == 0, lib.fcb_last_error().decode()
            got = out.cpu().numpy()
            assert np.array_equal(got, want), (npatches, call, got, want)


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
