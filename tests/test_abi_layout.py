"""The ctypes mirrors of the C ABI's structs (qlassical_b200._lib) have the
header's sizes and field offsets: a C program compiled here against
include/qlassical_b200.h prints them with sizeof/offsetof."""
import ctypes
import os
import shutil
import subprocess

import pytest

from qlassical_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "qlb_pool_view": _lib.PoolView,
    "qlb_exec_stats": _lib.ExecStats,
    "qlb_batch_tune_class": _lib.BatchTuneClass,
    "qlb_batch_info": _lib.BatchInfo,
    "qlb_server_config": _lib.ServerConfig,
    "qlb_server_info": _lib.ServerInfo,
    "qlb_request_info": _lib.RequestInfo,
    "qlb_check64_result": _lib.Check64Result,
    "qlb_transpile_config": _lib.TranspileConfig,
}


def c_layout(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "qlassical_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            if f[0].startswith("pad"):
                continue
            lines.append(f'    printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_struct_layouts_match_the_header(tmp_path):
    c = c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert c[(cname, "size")] == ctypes.sizeof(py), cname
        for f in py._fields_:
            if f[0].startswith("pad"):
                continue
            assert c[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
