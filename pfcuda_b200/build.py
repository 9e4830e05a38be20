"""Build libpfb200.so in-tree with nvcc for sm_100a.

    python -m pfcuda_b200.build [--verbose]

Each .cu file under csrc/ is compiled to an object in csrc/_build/ (only when
its sources changed) and linked into pfcuda_b200/libpfb200.so next to this file.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libpfb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


TUNE_JSON = os.path.join(HERE, "tune_table.json")
TUNE_H = os.path.join(CSRC, "tune_table.h")
_PANEL = {"registers": 1, "half_shared": 2, 1: 1, 2: 2}
_EPI = {"roundtrip": 1, "reduce": 2, "direct": 3, 1: 1, 2: 2, 3: 3}


def write_tune_header() -> str:
    """csrc/tune_table.h from tune_table.json (rewritten only when it changes)."""
    import json
    with open(TUNE_JSON) as f:
        t = json.load(f)
    d = t["defaults"]
    rows = []
    for e in t["entries"]:
        rows.append("    {%d, %d, %d, %d, %dLL, %dLL, %d, %d, %d, %d},  // %s" % (
            1 if e["dtype"] == "complex" else 0, 1 if e["mode"] == "split" else 0, e["n_min"], e["n_max"],
            e["batch_min"], e["batch_max"], _PANEL[e["panel"]], e["slices"], e["ranges"],
            _EPI[e.get("epilogue", d["epilogue"])], e.get("note", "")))
    body = "\n".join(rows) if rows else "    {-1, -1, 0, 0, 0LL, 0LL, 0, 0, 0, 0},  // (no measured entries)"
    text = f"""// tune_table.h -- generated by pfcuda_b200/build.py from pfcuda_b200/tune_table.json
// (the table pfcuda_b200/tune.py measures); do not edit.
#pragma once
#include <stdint.h>

#include "../../include/pfb200.h"

namespace pfb {{

struct TuneEntry {{
    int cplx, split, n_min, n_max;
    long long batch_min, batch_max;
    int panel, slices, ranges, epilogue;
}};

static const TuneEntry kTuneTable[] = {{
{body}
}};

// The first entry for this dtype class and mode whose order and batch bins
// hold (n, batch), else the defaults.
inline pfb_slog_config tuned_config(int dtype, int n, int64_t batch, bool split)
{{
    const int cplx = (dtype == PFB_C64 || dtype == PFB_C128) ? 1 : 0;
    for (const TuneEntry &e : kTuneTable)
        if (e.cplx == cplx && e.split == (split ? 1 : 0) && n >= e.n_min && n <= e.n_max &&
            batch >= e.batch_min && batch <= e.batch_max)
            return pfb_slog_config{{e.panel, e.slices, e.ranges, e.epilogue}};
    return pfb_slog_config{{{_PANEL[d["panel"]]}, {d["slices"]}, {d["ranges"]}, {_EPI[d["epilogue"]]}}};
}}

}}  // namespace pfb
"""
    old = open(TUNE_H).read() if os.path.exists(TUNE_H) else None
    if old != text:
        with open(TUNE_H, "w") as f:
            f.write(text)
    return TUNE_H


def _deps():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(p) for p in [src] + _deps())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, ""
    cmd = [_nvcc()] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    write_tune_header()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
