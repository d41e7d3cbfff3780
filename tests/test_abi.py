"""C-ABI checks that need no GPU: the library loads and exports every entry point
declared in include/fmm_b200.h, the ctypes structs match, and the product
refuses to run without a device instead of falling back to the CPU."""
import ctypes as C
import os
import re

import pytest

import fastmultipole_b200 as fm
from fastmultipole_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^FMM_API\s+[\w\s\*]+?\b(fmm_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
        assert n in L.SIGNATURES, n


def test_default_options_match_reference_defaults():
    o = L.default_options()
    # fmm! defaults (src/fmm.jl:862-923)
    assert o.expansion_order == 5 and o.leaf_size_source == 20 and abs(o.multipole_acceptance - 0.4) < 1e-15
    assert o.shrink_recenter == 1 and o.list_method == L.FMM_LIST_SELF_TUNING_TREE_STOP
    assert (o.scalar_potential, o.gradient, o.hessian) == (0, 1, 0)
    assert (o.farfield, o.nearfield, o.self_induced) == (1, 1, 1)


def test_struct_layouts_match_the_header(tmp_path):
    """Compile a probe against include/fmm_b200.h and compare sizes/offsets with the ctypes mirrors."""
    import subprocess
    structs = {"fmm_options": L.Options, "fmm_source_system": L.SourceSystem, "fmm_target_system": L.TargetSystem,
               "fmm_result": L.Result, "fmm_tree_view": L.TreeView, "fmm_request": L.Request}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "fmm_b200.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = dict(l.split() for l in subprocess.check_output([str(exe)]).decode().splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_cpu_fallback_without_device():
    with pytest.raises(fm.FMMError) as e:
        fm.Context(0)
    assert e.value.status == L.FMM_ERR_NO_DEVICE
