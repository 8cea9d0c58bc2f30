"""ASCII output frames (fcb_output_ascii) in the reference's fort.t / fort.q
format (fclaw2d_clawpatch46_fort_header_ascii, _fort_write_grid_header,
_fort_output_ascii).  The expected text is rebuilt here from the Fortran edit
descriptors with exact decimal arithmetic, independently of the library's
formatter, and every written value must read back to the state's 16
significant digits."""
from decimal import ROUND_HALF_EVEN, Decimal, localcontext

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def fortran_e(x: float, w: int, d: int) -> str:
    """Ew.d as gfortran writes it: [-]0.d1..dd E+xx (or +xxx for |exp| > 99)."""
    if x == 0.0:
        body = "0." + "0" * d + "E+00"
        return body.rjust(w)
    with localcontext() as ctx:
        ctx.prec = 1000  # exact: a double has at most 767 significant decimal digits
        v = Decimal(abs(x))
        e = v.adjusted() + 1  # x = 0.d1d2... * 10^e
        mant = (v.scaleb(-e)).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
        if mant >= 1:  # rounding carried into a new digit
            e += 1
            mant = (v.scaleb(-e)).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
        digits = f"{mant:.{d}f}"[2:]
    ex = f"E{'-' if e < 0 else '+'}{abs(e):02d}" if abs(e) <= 99 else f"{'-' if e < 0 else '+'}{abs(e):03d}"
    body = ("-" if x < 0 else "") + "0." + digits + ex
    return body.rjust(w)


def test_fortran_e_reference_points():
    assert fortran_e(1.0, 26, 16) == "    0.1000000000000000E+01"
    assert fortran_e(-2.5, 24, 16) == " -0.2500000000000000E+01"
    assert fortran_e(0.0, 30, 20) == "    0.00000000000000000000E+00"


def test_ascii_frame_matches_the_reference_format(gpu_lib, tmp_path):
    import forestclaw_b200 as fcb

    cfg = cases.radialdam_amr(seed=1, minlevel=2, maxlevel=3, mx=8, tfinal=0.05)
    d = fcb.Solver(cases.to_options(cfg))
    d.initialize()
    d.advance_all_levels(0.0, 0.9 / (8 * 4) / 1.5)
    d.output_ascii(3, str(tmp_path))
    q = d.get_q()
    leaves = d.leaves()
    t = (tmp_path / "fort.t0003").read_text().splitlines()
    assert t == [fortran_e(d.curr_time, 30, 20) + "    time",
                 f"{3:5d}                 meqn",
                 f"{len(leaves):5d}                 ngrids",
                 f"{0:5d}                 num_aux",
                 f"{2:5d}                 num_dim"]
    lines = (tmp_path / "fort.q0003").read_text().split("\n")
    k = 0
    mx = my = cfg.mx
    mbc = cfg.mbc
    for p, (lv, x, y) in enumerate(leaves):
        assert lines[k] == f"{p:5d}                 grid_number"
        assert lines[k + 1] == f"{lv:5d}                 AMR_level"
        assert lines[k + 2] == f"{0:5d}                 block_number"
        assert lines[k + 3] == f"{0:5d}                 mpi_rank"
        assert lines[k + 4] == f"{mx:5d}                 mx"
        assert lines[k + 5] == f"{my:5d}                 my"
        xl = x / float(1 << 28)
        yl = y / float(1 << 28)
        dx = (((x + (1 << (28 - lv))) / float(1 << 28)) - xl) / mx
        assert lines[k + 6] == fortran_e(xl, 24, 16) + "    xlow"
        assert lines[k + 7] == fortran_e(yl, 24, 16) + "    ylow"
        assert lines[k + 8] == fortran_e(dx, 24, 16) + "    dx"
        assert lines[k + 10] == ""
        k += 11
        for j in range(my):
            for i in range(mx):
                vals = [q[p, m, j + mbc, i + mbc] for m in range(3)]
                want = "".join(fortran_e(0.0 if abs(v) < 1e-99 else float(v), 26, 16) for v in vals)
                assert lines[k] == want, (p, i, j)
                back = [float(lines[k][26 * m:26 * (m + 1)]) for m in range(3)]
                assert np.allclose(back, vals, rtol=1e-15, atol=1e-99)
                k += 1
            assert lines[k] == "  "
            k += 1
    assert lines[k:] == [""]
