"""Every structure of the C ABI (include/halloc_c.h) has, in the Python
binding, the size and field offsets the C compiler gives it: the header is
compiled here with the host compiler and its offsetof() values compared
with ctypes'.  CPU only."""
import ctypes
import os
import subprocess

import pytest

import halloc_b200 as H
from halloc_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (ctypes class, C type, {ctypes field name: C field name} where they differ)
STRUCTS = [
    (H._COpts, "ha_opts_c", {}),
    (H._CStats, "ha_stats_t", {}),
    (H._CDump, "ha_state_dump_t", {}),
    (H._CPhaseResult, "ha_phase_result_t", {}),
    (H._CPhaseRefResult, "ha_phase_ref_result_t", {}),
    (H._CLatency, "ha_latency_stats_t", {}),
    (W._CPlan, "ha_batch_plan_t", {}),
    (H._CServeCfg, "ha_serve_cfg_t", {"lam": "lambda"}),
    (H._CServeResult, "ha_serve_result_t", {}),
]


@pytest.fixture(scope="module")
def c_layouts(tmp_path_factory):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "halloc_c.h"',
             'int main(void) {']
    for cls, cname, ren in STRUCTS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            cf = ren.get(f, f)
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {cf}));')
    lines += ['  return 0;', '}']
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True,
                               check=True).stdout.splitlines():
        cname, field, val = line.split()
        out[(cname, field)] = int(val)
    return out


@pytest.mark.parametrize("cls,cname,ren", STRUCTS, ids=[s[1] for s in STRUCTS])
def test_ctypes_layout_matches_c(c_layouts, cls, cname, ren):
    assert ctypes.sizeof(cls) == c_layouts[(cname, "size")]
    for f, _ in cls._fields_:
        assert getattr(cls, f).offset == c_layouts[(cname, f)], f
