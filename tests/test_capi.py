"""The C ABI library loads, exports every entry point the header declares,
and its options struct has the header's layout.  No GPU is needed."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "fclaw_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fcb_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def built():
    from forestclaw_b200 import build

    build.build()
    import forestclaw_b200 as fcb

    return fcb


def test_library_exports_every_declared_symbol(built):
    lib = built.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(built.EXPORTED_SYMBOLS)
    assert lib.fcb_abi_version() == 1


def test_options_layout_matches_header(built, tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "fclaw_b200.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu\\n\", sizeof(fcb_options_t),"
        " offsetof(fcb_options_t, refine_threshold), offsetof(fcb_options_t, problem_params),"
        " sizeof(fcb_counters_t)); printf(\"%zu %zu %zu\\n\", offsetof(fcb_options_t, step_variant),"
        " offsetof(fcb_options_t, precision), offsetof(fcb_options_t, macro_graph));"
        " printf(\"%zu %zu %zu\\n\", offsetof(fcb_options_t, dry_tolerance),"
        " offsetof(fcb_options_t, time_sync), offsetof(fcb_options_t, by));"
        " printf(\"%zu %zu\\n\", offsetof(fcb_options_t, weighted_partition),"
        " offsetof(fcb_options_t, ghost_fusion)); printf(\"%zu\\n\", offsetof(fcb_options_t, src_term));"
        " return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    from forestclaw_b200 import _Counters, _Options

    assert int(out[0]) == ctypes.sizeof(_Options)
    assert int(out[1]) == _Options.refine_threshold.offset
    assert int(out[2]) == _Options.problem_params.offset
    assert int(out[3]) == ctypes.sizeof(_Counters)
    assert int(out[4]) == _Options.step_variant.offset
    assert int(out[5]) == _Options.precision.offset
    assert int(out[6]) == _Options.macro_graph.offset
    assert int(out[7]) == _Options.dry_tolerance.offset
    assert int(out[8]) == _Options.time_sync.offset
    assert int(out[9]) == _Options.by.offset
    assert int(out[10]) == _Options.weighted_partition.offset
    assert int(out[11]) == _Options.ghost_fusion.offset
    assert int(out[12]) == _Options.src_term.offset


def test_invalid_options_rejected_before_any_device_call(built):
    o = built.Options(mx=12, my=12)
    with pytest.raises(built.FcbError) as e:
        built.Solver(o)
    assert e.value.code == 1  # FCB_ERR_INVALID
    o = built.Options(mthbc=(0, 1, 1, 1))
    with pytest.raises(built.FcbError) as e:
        built.Solver(o)
    assert e.value.code == 1
    # the mixed-precision update exists in the pipelined step form only
    for variant in (1, 2):
        o = built.Options(precision=built.PRECISION_MIXED, step_variant=variant)
        with pytest.raises(built.FcbError) as e:
            built.Solver(o)
        assert e.value.code == 1
    with pytest.raises(built.FcbError) as e:
        built.Solver(built.Options(precision=2))
    assert e.value.code == 1


def test_null_arguments_are_errors(built):
    lib = built.lib()
    assert lib.fcb_context_create(None, None, None) == 1
    assert b"null" in lib.fcb_last_error()


def test_forest_morton_key_matches_bit_loop(tmp_path):
    """The forest's z-order key (bit spreading) equals the key built bit by
    bit (x in the even bits, y in the odd bits of the low 28 bits)."""
    src = tmp_path / "mk.cpp"
    src.write_text(
        '#include <cstdio>\n#include <random>\n#include "fcb_forest.hpp"\n'
        "static uint64_t loop(int32_t x, int32_t y) { uint64_t k = 0;\n"
        "  for (int b = 0; b < 28; ++b) { k |= (uint64_t)((x >> b) & 1) << (2 * b);\n"
        "    k |= (uint64_t)((y >> b) & 1) << (2 * b + 1); } return k; }\n"
        "int main() { std::mt19937 g(7); int bad = 0;\n"
        "  const int32_t edge[] = {0, 1, 2, 3, (1 << 27) - 1, 1 << 27, (1 << 28) - 1};\n"
        "  for (int32_t a : edge) for (int32_t b : edge) bad += fcb::QuadForest::morton(a, b) != loop(a, b);\n"
        "  for (int k = 0; k < 200000; ++k) { int32_t x = g() & ((1 << 28) - 1), y = g() & ((1 << 28) - 1);\n"
        "    bad += fcb::QuadForest::morton(x, y) != loop(x, y); }\n"
        '  std::printf("%d\\n", bad); return 0; }\n')
    exe = tmp_path / "mk"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "forestclaw_b200" / "csrc"), str(src), "-o", str(exe)],
                   check=True)
    assert subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip() == "0"


def test_capacity_options_are_checked():
    """Capacity (mcapa > 0) belongs to the manifold advection solver, whose
    update exists in the four-barrier FP64 form (clawpack 4.6 and 5); other
    combinations fail at context creation (no device touched)."""
    import cases
    import forestclaw_b200 as fcb
    import oracle as O

    good = cases.to_options(O.filament_regression(4))
    for ok in (good, cases.to_options(O.filament_regression(5))):
        s = fcb.Solver(ok)
        del s
    for change in (dict(mcapa=0), dict(precision=1), dict(maux=2), dict(step_variant=3),
                   dict(problem=O.PERIODIC_DISC)):
        opts = cases.to_options(O.filament_regression(4))
        for k, v in change.items():
            setattr(opts, k, v)
        with pytest.raises(fcb.FcbError):
            fcb.Solver(opts)
    dam = cases.to_options(cases.radialdam_amr(seed=0, minlevel=2, maxlevel=3, mx=16))
    dam.mcapa = 1
    with pytest.raises(fcb.FcbError):
        fcb.Solver(dam)
