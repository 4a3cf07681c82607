"""The ctypes mirror of the C ABI must lay out every struct exactly as the C compiler does from
include/fslbm.h: same size and the same offset for every field (a mismatch would pass wrong
values across the boundary silently). Compiled with gcc on the host; no GPU needed."""
import ctypes
import os
import subprocess

import pytest

import flowcontrast_b200 as fb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = {  # C type -> Python mirror
    "fslbm_domain": fb.Domain, "fslbm_params": fb.Params, "fslbm_monitor": fb.Monitor,
    "fslbm_info": fb.Info, "fslbm_server_config": fb.ServerConfig,
    "fslbm_init_spec": fb.InitSpec, "fslbm_request": fb.Request, "fslbm_result": fb.Result,
    "fslbm_server_stats": fb.ServerStats,
}


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fslbm.h"', "int main(void) {"]
    for ctype, py in MIRRORS.items():
        lines.append(f'  printf("{ctype} sizeof %zu\\n", sizeof({ctype}));')
        for name, _ in py._fields_:
            lines.append(f'  printf("{ctype} {name} %zu\\n", offsetof({ctype}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        ctype, field, value = line.split()
        got[(ctype, field)] = int(value)
    return got


def test_ctypes_mirror_matches_c_layout(tmp_path):
    try:
        got = c_layout(tmp_path)
    except FileNotFoundError:
        pytest.skip("gcc is not available")
    for ctype, py in MIRRORS.items():
        assert ctypes.sizeof(py) == got[(ctype, "sizeof")], ctype
        for name, _ in py._fields_:
            assert getattr(py, name).offset == got[(ctype, name)], (ctype, name)
