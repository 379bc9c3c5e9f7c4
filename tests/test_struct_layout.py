"""CPU tests of the structures passed across the C ABI by value or by
pointer: the ctypes mirrors in tflows_b200/batch.py must match the C
layouts of include/tf_krylov.h field for field (a C program built with gcc
prints the compiler's offsets and sizes).  Also the bench's sweep-timeline
summary on a synthetic trace."""
import ctypes
import os
import subprocess

import pytest

from conftest import ROOT
from tflows_b200 import batch

STRUCTS = {
    "tf_batch_opts": (batch.BatchOpts, ["vec_fp32", "val_fp32", "sweep_iters", "max_systems",
                                        "ru_delta", "mem_budget", "two_phase_rows"]),
    "tf_batch_sweep": (batch.SweepRec, ["active", "items", "rows", "nnz", "iter_bytes", "ms",
                                        "kernel_ms"]),
}


@pytest.fixture(scope="module")
def c_layouts(tmp_path_factory):
    d = tmp_path_factory.mktemp("layout")
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "tf_krylov.h"',
           "int main(void) {"]
    for name, (_, fields) in STRUCTS.items():
        src.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for f in fields:
            src.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    src += ["  return 0;", "}"]
    c = d / "layout.c"
    c.write_text("\n".join(src) + "\n")
    exe = d / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(c), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        name, key, val = line.split()
        table[(name, key)] = int(val)
    return table


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_ctypes_mirror_matches_the_header(c_layouts, name):
    cls, fields = STRUCTS[name]
    assert ctypes.sizeof(cls) == c_layouts[(name, "size")]
    assert [f[0] for f in cls._fields_] == fields
    for f in fields:
        assert getattr(cls, f).offset == c_layouts[(name, f)], f


def test_trace_deciles_on_a_synthetic_trace():
    import bench
    kern = {k: 0.0 for k in batch.KERNELS}
    trace = [dict(active=10 - k, items=100 - 5 * k, rows=1000 - 50 * k, nnz=7000 - 350 * k,
                  iter_bytes=1.0e9, ms=2.0, kernel_ms=dict(kern)) for k in range(10)]
    d = bench._trace_deciles(trace, 4)
    assert len(d) == 10
    assert [x["running"] for x in d] == list(range(10, 0, -1))
    assert d[0]["at_ms"] == 0.0 and d[1]["at_ms"] == 2.0
    # 8 iterations of 1 GB in 2 ms
    assert d[0]["gbs_if_all_iterate"] == pytest.approx(4000.0)
    assert "kernel_ms" not in d[0]
    profiled = [dict(t, kernel_ms=dict(kern, spmv=1.0)) for t in trace]
    p = bench._trace_deciles(profiled, 4)
    assert p[0]["spmv_gbs_if_all_iterate"] > 0 and p[0]["kernel_ms"]["spmv"] == 1.0
    assert bench._trace_deciles([], 4) == []
