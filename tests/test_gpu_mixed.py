"""Mixed FP32/FP64 update against the FP64 oracle.

The mixed form computes Riemann solves, limiters, transverse parts and ghost
interpolation in FP32, and the flux sums, the cell update, the state and the
mass sums in FP64.  Its contract: relative L1 error <= 1e-5 against the FP64
oracle on the same mesh; max error and mass drift are measured and bounded too.
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

L1_TOL = 1e-5      # relative L1 error, interior cells, all components
MAX_TOL = 1e-4     # relative max-norm error
MASS_TOL = 1e-6    # relative mass drift vs the FP64 oracle


def _pair(cfg):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cfg)
    opts.precision = fcb.PRECISION_MIXED
    o = O.OracleSolver(cfg)
    d = fcb.Solver(opts)
    o.initialize()
    d.initialize()
    return o, d


def _errors(qd, qo, mbc):
    a = qd[..., mbc:-mbc, mbc:-mbc]
    b = qo[..., mbc:-mbc, mbc:-mbc]
    diff = np.abs(a - b)
    l1 = float(diff.sum() / max(np.abs(b).sum(), 1e-300))
    mx = float(diff.max() / max(1.0, np.abs(b).max()))
    return l1, mx


def _mass_drift(d, o):
    """Largest component difference of the conserved sums, relative to the
    largest sum (momentum sums may be zero by symmetry)."""
    m_d, m_o = np.asarray(d.conservation_check()), np.asarray(o.conservation())
    return float(np.max(np.abs(m_d - m_o)) / max(float(np.max(np.abs(m_o))), 1e-300))


def test_mixed_swirl_plain_method_case(gpu_lib):
    """Uniform level 4 (256 patches), mx = 16, 200 steps of dt = 0.9/256."""
    cfg = cases.swirl_uniform(level=4, mx=16)
    dt = cases.swirl_dt(level=4, mx=16)
    o, d = _pair(cfg)
    t = 0.0
    for _ in range(200):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
    l1, mx = _errors(d.get_q(), o.all_q(), cfg.mbc)
    assert l1 <= L1_TOL, f"L1 {l1:.3e}"
    assert mx <= MAX_TOL, f"max {mx:.3e}"
    assert abs(c_d - c_o) <= 1e-6 * c_o
    assert _mass_drift(d, o) <= MASS_TOL


@pytest.mark.parametrize("mx", [16, 32])
def test_mixed_radialdam(gpu_lib, mx):
    cfg = cases.radialdam_uniform(level=2, mx=mx)
    dt = 0.4 / (mx * 4) / 1.5
    o, d = _pair(cfg)
    t = 0.0
    for _ in range(40):
        o.advance(t, dt)
        d.advance_all_levels(t, dt)
        t += dt
    l1, mx_err = _errors(d.get_q(), o.all_q(), cfg.mbc)
    assert l1 <= L1_TOL, f"L1 {l1:.3e}"
    assert mx_err <= MAX_TOL, f"max {mx_err:.3e}"
    assert _mass_drift(d, o) <= MASS_TOL


def test_mixed_quadrants(gpu_lib):
    cfg = cases.quadrants_uniform(level=2, mx=16)
    dt = 0.3 / (16 * 4) / 2.0
    o, d = _pair(cfg)
    t = 0.0
    for _ in range(30):
        o.advance(t, dt)
        d.advance_all_levels(t, dt)
        t += dt
    l1, mx_err = _errors(d.get_q(), o.all_q(), cfg.mbc)
    assert l1 <= L1_TOL, f"L1 {l1:.3e}"
    assert mx_err <= MAX_TOL, f"max {mx_err:.3e}"
    assert _mass_drift(d, o) <= MASS_TOL


def test_mixed_amr_subcycled_with_fp32_interpolation(gpu_lib):
    """AMR shallow water on a fixed refined mesh: subcycling, time interpolation
    and FP32 coarse-to-fine ghost interpolation, compared patch by patch."""
    cfg = cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=16, tfinal=0.05)
    o, d = _pair(cfg)
    assert d.leaves() == o.leaves()
    t, dt = 0.0, 0.9 / (16 * 4) / 1.5
    for _ in range(4):
        o.advance(t, dt)
        d.advance_all_levels(t, dt)
        t += dt
    l1, mx_err = _errors(d.get_q(), o.all_q(), cfg.mbc)
    assert l1 <= L1_TOL, f"L1 {l1:.3e}"
    assert mx_err <= MAX_TOL, f"max {mx_err:.3e}"
    assert _mass_drift(d, o) <= MASS_TOL


def _central(leaves, level):
    n = 1 << level
    return [k for k, (lv, x, y) in enumerate(leaves)
            if 2 <= (x >> (28 - lv)) <= n - 3 and 2 <= (y >> (28 - lv)) <= n - 3]


def test_mixed_geoclaw_pulse_amr(gpu_lib):
    """GeoClaw f-waves over bathymetry, subcycled levels 2-4 with FP32 ghost
    interpolation: the state against the FP64 oracle within the contract, and
    the pulse itself (q - q0, amplitude 0.05) to 1e-3 of its own L1 norm."""
    cfg = cases.bathy_lake(minlevel=2, maxlevel=4, mx=16, seed=2, amp=0.05)
    o, d = _pair(cfg)
    q0 = o.all_q()
    t, dt = 0.0, 0.5 / (16 * 4)
    for k in range(3):
        o.advance(t, dt)
        d.advance_all_levels(t, dt)
        t += dt
    qd, qo = d.get_q(), o.all_q()
    l1, mx = _errors(qd, qo, cfg.mbc)
    assert l1 <= L1_TOL and mx <= MAX_TOL, (l1, mx)
    m = cfg.mbc
    pert = np.abs(qo - q0)[..., m:-m, m:-m].sum()
    assert np.abs(qd - qo)[..., m:-m, m:-m].sum() <= 1e-3 * pert
    assert _mass_drift(d, o) <= MASS_TOL


def test_mixed_geoclaw_lake_at_rest(gpu_lib):
    """The hydrostatic part stays FP64, so a lake at rest stays at rest to
    FP64 round-off in the mixed form too (uniform level, central patches)."""
    cfg = cases.bathy_lake(level=3, mx=16, amp=0.0)
    o, d = _pair(cfg)
    q0 = d.get_q()
    dt = 0.5 / (16 * 8)
    for k in range(10):
        d.advance_all_levels(k * dt, dt)
    inner = _central(d.leaves(), 3)
    dq = np.abs(d.get_q() - q0)[inner][:, :, 2:-2, 2:-2]
    assert float(dq.max()) <= 1e-14, f"lake-at-rest residual {dq.max():.3e}"
