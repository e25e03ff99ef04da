"""CPU tests of the C-ABI library: it loads, exports every declared symbol, and
its host-only entry points behave (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fame.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^FAME_API\s+(?:int|long long|const char\*)\s+(fame_\w+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    from fame_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    from fame_b200 import _lib
    names = set(_declared())
    bound = set(_lib.SIGNATURES) | {"fame_status_string", "fame_last_error", "fame_kernel_launches"}
    assert names <= bound, names - bound


def test_status_strings_and_default_opts():
    from fame_b200 import _lib
    L = _lib.lib
    assert L.fame_status_string(0) == b"FAME_OK"
    assert L.fame_status_string(7) == b"FAME_ERR_SINGULAR"
    o = _lib.fame_krinv_opts()
    assert L.fame_krinv_default_opts(C.byref(o)) == 0
    assert o.tolCG == 1e-10 and o.maxitCG == 1200 and o.tolM == 1e-12 and o.maxitKr == 600
    assert o.epsC == 4.0 and o.useKrPreconditioner == 1 and o.mhatPreconditioner == 1
    assert o.tolInner32 == 3e-6 and o.refineTarget == 0.1
    assert L.fame_version() >= 100


def test_null_arguments_are_rejected_without_gpu():
    from fame_b200 import _lib
    L = _lib.lib
    assert L.fame_krinv_default_opts(None) == 1
    assert L.fame_mass_apply(None, 0, None, None, 1, 0) == 1
    assert b"FAME_ERR_INVALID" in L.fame_last_error()
    assert L.fame_krinv_apply(None, None, None, 1) == 1
    assert L.fame_basis_get(None, 0, None) == 1


def test_method_a_entry_points_reject_bad_arguments_without_gpu():
    from fame_b200 import _lib
    L = _lib.lib
    out = C.c_void_p()
    assert L.fame_osi_create(None, None, 1e-4, 1e-4, 1e-10, 100, C.byref(out)) == 1
    assert b"fame_osi_create" in L.fame_last_error()
    assert L.fame_osi_apply(None, None, None, 1) == 1
    lam = (C.c_double * 1)()
    assert L.fame_osi_eigs(None, 1, 1e-8, 10, 20, None, lam, None, None) == 1
    assert L.fame_osi_stats_get(None, None) == 1
    assert L.fame_apply_K_original(None, None, None, 1) == 1
    assert L.fame_osi_destroy(None) == 0


def test_struct_layouts_match_header(tmp_path):
    """Every ABI struct of include/fame.h, compiled by the C compiler, has the size and field
    offsets of its ctypes mirror."""
    import shutil
    import subprocess
    from fame_b200 import _lib
    structs = [_lib.fame_krinv_opts, _lib.fame_krinv_stats, _lib.fame_basis_info, _lib.fame_osi_stats,
               _lib.fame_lanczos_info]
    cc = shutil.which("gcc") or shutil.which("cc")
    assert cc, "a C compiler is needed for the layout check"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fame.h"', "int main(void) {"]
    for st in structs:
        lines.append('printf("%%s %%zu\\n", "%s", sizeof(%s));' % (st.__name__, st.__name__))
        for f in st._fields_:
            lines.append('printf("%%s.%%s %%zu\\n", "%s", "%s", offsetof(%s, %s));'
                         % (st.__name__, f[0], st.__name__, f[0]))
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                           check=True).stdout.splitlines())
    for st in structs:
        assert int(got[st.__name__]) == C.sizeof(st), st.__name__
        for f in st._fields_:
            assert int(got["%s.%s" % (st.__name__, f[0])]) == getattr(st, f[0]).offset, (st.__name__, f[0])


def test_twiddle_header_is_generated_and_exact():
    import importlib.util
    import math
    pkg = os.path.join(ROOT, "null--space-free-6d-projection-method_b200", "csrc")
    txt = open(os.path.join(pkg, "twiddles.cuh")).read()
    vals = dict(re.findall(r"case (\d+): return ([-0-9.e]+);", txt.split("tw_sin")[0]))
    assert float(vals[str(5 * 32 + 1)]) == math.cos(2 * math.pi / 5) or \
        abs(float(vals[str(5 * 32 + 1)]) - math.cos(2 * math.pi / 5)) < 1e-16
    assert float(vals[str(3 * 32 + 1)]) == -0.5
    # every length up to 27 (the rank-1 FFT radices), within a few ulps of libm on a rounded argument
    for n in range(1, 28):
        for e in range(n):
            assert abs(float(vals[str(n * 32 + e)]) - math.cos(2 * math.pi * e / n)) < 2e-15, (n, e)


def test_mex_gateway_compiles_against_the_c_abi():
    """mex/fame_mex.c type-checks against include/fame.h (MATLAB's API declared by stubs)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    src = os.path.join(ROOT, "null--space-free-6d-projection-method_b200", "mex", "fame_mex.c")
    r = subprocess.run([gcc, "-std=c99", "-fsyntax-only", "-Wall", "-Wextra", "-Wno-unused-parameter", "-Werror",
                        "-I", os.path.join(ROOT, "tests", "mex_stub"), "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
