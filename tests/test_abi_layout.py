"""The ctypes mirrors of the C structs have the C layouts: gcc compiles a
probe against include/psod.h and oracle/psod_oracle.h that prints every
struct's size and each field's offset, and the Python side must agree."""

import ctypes as C
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from psod_b200 import capi  # noqa: E402

PAIRS = [
    ("psod_params", capi.Params, "psod.h"),
    ("psod_halo_table", capi.HaloTable, "psod.h"),
    ("psod_run_stats", capi.RunStats, "psod.h"),
    ("psod_train_params", capi.TrainParams, "psod.h"),
    ("psod_tuning", capi.Tuning, "psod.h"),
    ("psod_fof_params", capi.FofParams, "psod.h"),
    ("psod_fof_stats", capi.FofStats, "psod.h"),
    ("psod_fof_table", capi.FofTable, "psod.h"),
    ("psod_props_params", capi.PropsParams, "psod.h"),
    ("psod_props_stats", capi.PropsStats, "psod.h"),
    ("psod_props_table", capi.PropsTable, "psod.h"),
    ("psod_oracle_params", O._Params, "psod_oracle.h"),
    ("psod_oracle_result", O._Result, "psod_oracle.h"),
    ("psod_oracle_audit", O._Audit, "psod_oracle.h"),
    ("psod_oracle_fof_params", O._FofParams, "psod_oracle_fof.h"),
    ("psod_oracle_fof_result", O._FofResult, "psod_oracle_fof.h"),
    ("psod_oracle_props_params", O._PropsParams, "psod_oracle_props.h"),
    ("psod_oracle_props_out", O._PropsOut, "psod_oracle_props.h"),
]


def _probe_source() -> str:
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "psod.h"', '#include "psod_oracle.h"',
             '#include "psod_oracle_fof.h"', '#include "psod_oracle_props.h"', "int main(void) {"]
    for cname, py, _ in PAIRS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in py._fields_:
            lines.append(f'  printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    return "\n".join(lines)


def test_ctypes_layouts_match_headers(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "probe.c"
    src.write_text(_probe_source())
    exe = tmp_path / "probe"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle"),
                    str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                              text=True).stdout.splitlines())
    for cname, py, _ in PAIRS:
        assert int(got[f"{cname} size"]) == C.sizeof(py), cname
        for fname, *_ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"
