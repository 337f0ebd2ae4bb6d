"""CPU: the ctypes mirrors of the C ABI structs (package `_lib`, `serving`)
have the header's sizes and field offsets.  A small C program built against
include/b200sssp.h prints sizeof / offsetof for every mirrored field; a
mismatch would make the Python layer read or pass shifted fields."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _pairs():
    from b200sssp import _lib, serving
    return {"b2_csr": _lib.CSR, "b2_graph_info": _lib.GraphInfo, "b2_sssp_opts": _lib.Opts,
            "b2_trace_entry": _lib.TraceEntry, "b2_progress": _lib.Progress, "b2_stats": _lib.Stats, "b2_host_csr": _lib.HostCSR,
            "b2_server_opts": serving.ServerOpts, "b2_completion": serving.Completion,
            "b2_server_info_t": serving.ServerInfo, "b2_load_opts": serving.LoadOpts,
            "b2_load_report": serving.LoadReport}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_header(tmp_path):
    pairs = _pairs()
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "b200sssp.h"', "int main(void) {"]
    for cname, py in pairs.items():
        src.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for name, *_ in py._fields_:
            src.append(f'  printf("{cname} {name} %zu\\n", offsetof({cname}, {name}));')
    src.append("  return 0;\n}")
    c_file, exe = tmp_path / "layout.c", tmp_path / "layout"
    c_file.write_text("\n".join(src))
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(c_file), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    mismatches = []
    for line in out.splitlines():
        cname, field, value = line.split()
        py = pairs[cname]
        got = C.sizeof(py) if field == "size" else getattr(py, field).offset
        if got != int(value):
            mismatches.append((cname, field, int(value), got))
    assert not mismatches
