"""Regenerate reference_prototypes.json: the C prototypes the reference's public
headers declare (include/{potrf,getrf,syrk,trsm,gemm,kernels}/*.h; benchmark and
utility headers excluded), as (return type, [(parameter type, parameter
name)], header path, line).  The ABI test checks this library's headers against
it: the same names, parameter order, parameter names and parameter types once
the documented type substitutions are applied.

    HDBF_REFERENCE_ROOT=<reference checkout> python tests/golden/make_prototypes.py

HDBF_REFERENCE_ROOT defaults to /root/reference.
"""
from __future__ import annotations

import glob
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("HDBF_REFERENCE_ROOT", "/root/reference")
DIRS = ("potrf", "getrf", "syrk", "trsm", "gemm", "kernels")


def strip_comments(src: str) -> str:
    # keep line numbers: replace comment text by the same number of newlines
    src = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    return re.sub(r"(?m)^\s*#[^\n]*", "", src)  # preprocessor lines


def split_param(p: str):
    p = " ".join(p.split())
    m = re.match(r"^(.*?[\s\*&])([A-Za-z_]\w*)$", p)
    if not m:
        return p, ""
    typ = m.group(1).replace(" *", "*").strip()
    return typ, m.group(2)


PROTO = re.compile(r"^\s*(void|int|float|double|size_t)\s+([A-Za-z_]\w*)\s*\(([^()]*)\)\s*$", re.S)


def prototypes(path: str):
    src = strip_comments(open(path).read())
    out = {}
    pos = 0
    for stmt in src.split(";"):
        start = pos
        pos += len(stmt) + 1
        cut = max(stmt.rfind("{"), stmt.rfind("}"))
        body = stmt[cut + 1:]
        m = PROTO.match(body)
        if not m:
            continue
        ret, name, params = m.group(1), m.group(2), m.group(3)
        offset = start + cut + 1 + m.start(2)
        line = src[:offset].count("\n") + 1
        plist = [split_param(p) for p in params.split(",") if p.strip() and p.strip() != "void"]
        out[name] = {"ret": ret, "params": plist, "file": os.path.relpath(path, REF), "line": line}
    return out


def main():
    allp = {}
    for d in DIRS:
        for h in sorted(glob.glob(os.path.join(REF, "include", d, "*.h"))):
            allp.update(prototypes(h))
    with open(os.path.join(HERE, "reference_prototypes.json"), "w") as f:
        json.dump(dict(sorted(allp.items())), f, indent=1)
    print(f"{len(allp)} prototypes")


if __name__ == "__main__":
    main()
