"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: the step, ghost and regrid kernels are compiled without FMA
contraction and follow the reference's operation order, so square roots and
divisions (correctly rounded on both sides) give identical bits; the swirl
velocities use sin(), whose last bit may differ between CUDA and glibc, so the
advection cases allow 1e-12 relative max-norm per step (the contract's bound).
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def _pair(cfg):
    import forestclaw_b200 as fcb

    o = O.OracleSolver(cfg)
    d = fcb.Solver(cases.to_options(cfg))
    o.initialize()
    d.initialize()
    return o, d


def _rel_err(a, b):
    scale = max(1.0, float(np.max(np.abs(b))))
    return float(np.max(np.abs(a - b))) / scale


def _assert_same_mesh(o, d):
    assert d.leaves() == o.leaves()


def _oracle_q(o):
    """Oracle patch arrays in the order fcb_get_q returns: (patch, m, j, i) for
    clawpack 4.6, (patch, j, i, m) for clawpack 5."""
    q = o.all_q()
    return np.moveaxis(q, 1, -1) if o.cfg.claw_version == 5 else q


def _pair_variant(cfg, variant):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cfg)
    opts.step_variant = variant
    o = O.OracleSolver(cfg)
    d = fcb.Solver(opts)
    o.initialize()
    d.initialize()
    return o, d


@pytest.mark.parametrize("variant", [1, 2, 3])
@pytest.mark.parametrize("mx", [8, 16, 32])
def test_uniform_swirl_steps(gpu_lib, mx, variant):
    """Every step-kernel form (CTA rows, warp-synchronous, pipelined CTA) against the oracle."""
    cfg = cases.swirl_uniform(level=3, mx=mx)
    dt = cases.swirl_dt(level=3, mx=mx)
    o, d = _pair_variant(cfg, variant)
    _assert_same_mesh(o, d)
    assert np.array_equal(d.get_q(), o.all_q()), "qinit differs"
    t = 0.0
    for step in range(12):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        err = _rel_err(d.get_q(), o.all_q())
        assert err <= REL_TOL, f"step {step}: rel err {err:.3e}"
        assert abs(c_d - c_o) <= 1e-12 * max(1.0, c_o), (c_d, c_o)


@pytest.mark.parametrize("variant", [1, 3])
@pytest.mark.parametrize("mx", [16, 32])
def test_uniform_radialdam_bit_exact(gpu_lib, mx, variant):
    cfg = cases.radialdam_uniform(level=2, mx=mx)
    dt = 0.4 / (mx * 4) / 1.5
    o, d = _pair_variant(cfg, variant)
    assert np.array_equal(d.get_q(), o.all_q())
    t = 0.0
    for step in range(10):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        qd, qo = d.get_q(), o.all_q()
        assert np.array_equal(qd, qo), f"step {step}: max diff {np.max(np.abs(qd - qo)):.3e}"
        assert c_d == c_o


@pytest.mark.parametrize("variant", [1, 3])
@pytest.mark.parametrize("mx", [8, 16])
def test_uniform_quadrants_bit_exact(gpu_lib, mx, variant):
    cfg = cases.quadrants_uniform(level=2, mx=mx)
    dt = 0.3 / (mx * 4) / 2.0
    o, d = _pair_variant(cfg, variant)
    assert np.array_equal(d.get_q(), o.all_q())
    t = 0.0
    for step in range(8):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        qd, qo = d.get_q(), o.all_q()
        assert np.array_equal(qd, qo), f"step {step}: max diff {np.max(np.abs(qd - qo)):.3e}"
        assert c_d == c_o


@pytest.mark.parametrize("solver", ["radialdam", "quadrants"])
@pytest.mark.parametrize("mx", [8, 64])
def test_cta_form_patch_sizes_and_partial_ctas(gpu_lib, solver, mx):
    """The four-barrier form packs 256 // (mx + 4) patches per CTA for the Roe
    systems (21 at mx = 8, 3 at mx = 64): 16 patches leave a partially filled
    last CTA; every array bit-identical to the oracle."""
    if solver == "radialdam":
        cfg, dt = cases.radialdam_uniform(level=2, mx=mx), 0.4 / (mx * 4) / 1.5
    else:
        cfg, dt = cases.quadrants_uniform(level=2, mx=mx), 0.3 / (mx * 4) / 2.0
    o, d = _pair_variant(cfg, 1)
    t = 0.0
    for step in range(4):
        assert o.advance(t, dt) == d.advance_all_levels(t, dt)
        t += dt
        assert np.array_equal(d.get_q(), o.all_q()), f"step {step}"


def test_single_step_update_protocol(gpu_lib):
    """patch_vt->single_step_update semantics: the batch runs on the last call."""
    cfg = cases.radialdam_uniform(level=2, mx=16)
    dt = 0.005
    o, d = _pair(cfg)
    n = d.num_patches
    cfls = [d.single_step_update(p, 0.0, dt, p, n) for p in range(n)]
    assert all(c == 0.0 for c in cfls[:-1])
    c_o = o.update_single_step(2, 0.0, dt)
    assert cfls[-1] == c_o
    assert np.array_equal(d.get_q(), o.all_q())


PIN_CONFIGS = {
    "swirl": O.swirl_regression, "quadrants": O.quadrants_regression,
    "quadrants_claw5": lambda: O.quadrants_regression(5),
    "bump": O.bump_regression, "bump_claw5": lambda: O.bump_regression(5),
    "periodic": O.periodic_regression, "periodic_claw5": lambda: O.periodic_regression(5),
    "filament": O.filament_regression, "filament_claw5": lambda: O.filament_regression(5),
}


@pytest.mark.parametrize("name", sorted(PIN_CONFIGS))
def test_regression_pins_on_gpu(gpu_lib, name):
    """The reference's own regression counters, reproduced by the CUDA path, with
    the final fields equal to the oracle's (bump: 24 advances and 14 new
    domains, its clawpack 5 run with solid walls, mthbc = 3 on all four sides;
    periodic: a 2 x 2 brick periodic in x and y, 8 / 601 / 8; filament: the
    cart-mapped 2 x 2 brick with capacity and the manifold solvers, 22 / 721 / 10)."""
    import json
    from pathlib import Path

    pins = json.loads((Path(__file__).parent / "golden" / "regression_pins.json").read_text())[name]["values"]
    cfg = PIN_CONFIGS[name]()
    # swirl velocities come from sin(), the bump's initial depth from exp(): CUDA
    # and glibc may differ in the last bit there; the Euler runs and the
    # periodic and filament bricks (sqrt and arithmetic only) are exact
    exact = name.startswith("quadrants") or name.startswith("periodic") or name.startswith("filament")
    tol = 0.0 if exact else 1e-11
    o, d = _pair(cfg)
    _assert_same_mesh(o, d)
    assert _rel_err(d.get_q(), _oracle_q(o)) <= (0.0 if exact else 1e-15)
    o.run()
    d.run()
    c = d.counters()
    assert c["count_amr_advance"] == pins["count_amr_advance"]
    assert d.num_patches == pins["global_num_patches"]
    assert c["count_amr_new_domain"] == pins["count_amr_new_domain"]
    _assert_same_mesh(o, d)
    err = _rel_err(d.get_q(), _oracle_q(o))
    assert err <= tol, f"rel err {err:.3e}"


def test_amr_radialdam_macro_steps(gpu_lib):
    """AMR shallow water with subcycling and time interpolation: advance + regrid
    step by step, comparing mesh and every patch array."""
    cfg = cases.radialdam_amr(seed=0, minlevel=2, maxlevel=4, mx=16, tfinal=0.05)
    o, d = _pair(cfg)
    _assert_same_mesh(o, d)
    assert np.array_equal(d.get_q(), o.all_q())
    t, dt = 0.0, 0.9 / (16 * 4) / 1.5
    for k in range(4):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        assert c_d == c_o
        qd, qo = d.get_q(), o.all_q()
        assert np.array_equal(qd, qo), f"macro step {k}: max diff {np.max(np.abs(qd - qo)):.3e}"
        t += dt
        o.regrid()
        d.regrid()
        _assert_same_mesh(o, d)
        assert np.array_equal(d.get_q(), o.all_q()), f"after regrid {k}"


def test_mass_conservation_matches_oracle(gpu_lib):
    cfg = cases.radialdam_uniform(level=2, mx=16)
    o, d = _pair(cfg)
    for k in range(5):
        o.advance(k * 0.002, 0.002)
        d.advance_all_levels(k * 0.002, 0.002)
    m_o, m_d = o.conservation(), d.conservation_check()
    assert np.allclose(m_d, m_o, rtol=1e-13, atol=1e-15)


def test_macro_step_graph_replays_bit_exact(gpu_lib):
    """advance_all_levels with the captured macro-step graph (subcycling, time
    interpolation, ghost fills) against issuing every launch from the host, on
    a refined mesh, and against the oracle."""
    import forestclaw_b200 as fcb

    cfg = cases.radialdam_amr(seed=2, minlevel=2, maxlevel=4, mx=16, tfinal=0.05)
    o = O.OracleSolver(cfg)
    o.initialize()
    solvers = []
    for graph in (0, 1):
        opts = cases.to_options(cfg)
        opts.macro_graph = graph
        opts.ghost_fusion = 1  # this mesh has one level: keep the graph path (fused steps launch directly)
        d = fcb.Solver(opts)
        d.initialize()
        solvers.append(d)
    eager, graphed = solvers
    assert eager.leaves() == graphed.leaves() == o.leaves()
    t, dt = 0.0, 0.9 / (16 * 4) / 1.5
    for k in range(5):
        c_o = o.advance(t, dt)
        c_e = eager.advance_all_levels(t, dt)
        c_g = graphed.advance_all_levels(t, dt)
        t += dt
        assert c_e == c_g == c_o
        qg, qe = graphed.get_q(), eager.get_q()
        assert np.array_equal(qg, qe), f"macro step {k}"
        assert np.array_equal(qg, o.all_q()), f"macro step {k}"
    ce, cg = eager.counters(), graphed.counters()
    assert cg["count_graph_replays"] == 3  # eager, capture, then replays
    assert ce["count_graph_replays"] == 0
    for name in ("count_single_step", "count_ghost_waves", "count_kernel_launches"):
        assert cg[name] == ce[name], name


@pytest.mark.parametrize("case", ["swirl", "radialdam"])
def test_autotuned_form_is_bit_identical_to_forced_form(gpu_lib, case):
    """step_variant 0 times the available step forms and ghost unrolls on
    scratch copies; the run must equal the same run with the chosen form forced,
    bit for bit (the tuner leaves the state alone and every form is exact)."""
    import forestclaw_b200 as fcb

    if case == "swirl":
        cfg, dt = cases.swirl_uniform(level=4, mx=16), cases.swirl_dt(level=4, mx=16)
    else:
        cfg, dt = cases.radialdam_uniform(level=3, mx=16), 0.4 / (16 * 8) / 1.5
    auto = fcb.Solver(cases.to_options(cfg))
    auto.initialize()
    assert auto.autotune_info()["step_form"] == 0
    t = 0.0
    for _ in range(4):
        auto.advance_all_levels(t, dt)
        t += dt
    info = auto.autotune_info()
    assert info["step_form"] in (1, 2, 3) and info["ghost_unroll"] in (2, 4, 8), info
    opts = cases.to_options(cfg)
    opts.step_variant = info["step_form"]
    forced = fcb.Solver(opts)
    forced.initialize()
    t = 0.0
    for _ in range(4):
        forced.advance_all_levels(t, dt)
        t += dt
    assert np.array_equal(auto.get_q(), forced.get_q())
    auto.close()
    forced.close()


def test_merged_level_launches_bit_exact(gpu_lib):
    """Subcycled macro steps on a mesh of several levels: with the macro-step
    table the level updates between two ghost updates go out as one launch
    (each patch reads its level's dt); they must equal one launch per level
    (macro_graph 0) and the oracle, through regrids."""
    import forestclaw_b200 as fcb

    cfg = cases.quadrants_amr(seed=1, minlevel=2, maxlevel=5, mx=8)
    o = O.OracleSolver(cfg)
    o.initialize()
    solvers = []
    for graph in (0, 2):
        opts = cases.to_options(cfg)
        opts.macro_graph = graph
        d = fcb.Solver(opts)
        d.initialize()
        solvers.append(d)
    per_level, merged = solvers
    assert len({lv for lv, _, _ in o.leaves()}) >= 2
    t, dt = 0.0, 0.9 / (8 * 32) / 1.5
    for k in range(4):
        c_o = o.advance(t, dt)
        assert per_level.advance_all_levels(t, dt) == c_o
        assert merged.advance_all_levels(t, dt) == c_o
        t += dt
        q = o.all_q()
        assert np.array_equal(per_level.get_q(), q), f"macro step {k}"
        assert np.array_equal(merged.get_q(), q), f"macro step {k}"
        o.regrid()
        per_level.regrid()
        merged.regrid()
        assert merged.leaves() == per_level.leaves() == o.leaves()
    cp, cm = per_level.counters(), merged.counters()
    assert cm["count_single_step"] == cp["count_single_step"]
    assert cm["count_kernel_launches"] < cp["count_kernel_launches"]


@pytest.mark.parametrize("case", ["swirl_fused", "amr_swe"])
def test_async_macro_steps_equal_sync(gpu_lib, case):
    """fcb_advance_all_levels_async enqueues the same macro steps as
    fcb_advance_all_levels without waiting for each CFL number; the running
    maximum that fcb_read_max_cfl returns equals the largest of the
    synchronous CFL numbers, bit for bit, and so do the fields (a mesh of one
    level with the ghost exchange fused into the step, and a subcycled AMR
    mesh with time interpolation, both with the macro-step graph)."""
    import forestclaw_b200 as fcb

    if case == "swirl_fused":
        cfg, dt = cases.swirl_uniform(level=4, mx=16), cases.swirl_dt(level=4, mx=16)
    else:
        cfg, dt = cases.radialdam_amr(seed=0, minlevel=2, maxlevel=4, mx=16), 0.004
    sync = fcb.Solver(cases.to_options(cfg))
    asyn = fcb.Solver(cases.to_options(cfg))
    sync.initialize()
    asyn.initialize()
    assert asyn.read_max_cfl() == 0.0
    cfls = [sync.advance_all_levels(k * dt, dt) for k in range(4)]
    for k in range(4):
        asyn.advance_all_levels_async(k * dt, dt)
    assert asyn.read_max_cfl() == max(cfls)
    assert asyn.read_max_cfl() == 0.0  # reset by the read
    assert np.array_equal(asyn.get_q(), sync.get_q())
    sync.close()
    asyn.close()
