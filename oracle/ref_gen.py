"""Extract the reference's own OpenCL functions for the host build of oracle/_ref.

TEST INFRASTRUCTURE ONLY (the parity checker's checker).  Reads the named functions,
kernels, macros and typedefs from the reference's .cl files where they lie and writes
them to <out>/*.inc, each item preceded by a #line directive naming its source file and
line, so compiler messages and debuggers point into the reference.  The text is kept
as written except for OpenCL syntax that C++ spells differently (ref_cl.h supplies
the rest):

* vector literals ``(float4)(a, b)`` and ``(float4){a, b}`` become ``make_float4(a, b)``;
* ``__local T name[N];`` inside a kernel becomes ``static T name[N];`` (the launcher runs
  one work-group at a time, so a function-static array is that group's local memory);
* ``__attribute__((reqd_work_group_size(...)))`` is dropped.

One edit goes beyond syntax, listed in PATCHES: getNonBond_GridFF_Bspline_ex2 has the
barrier that closes its tile loop commented out, so a work-item that starts the next tile
overwrites the __local tile while others still read it.  On a device that runs the 32-wide
work-group as one warp in lockstep the race never shows; the fiber launcher of ref_cl.h runs
work-items one after another between barriers, so the barrier is restored to give the
lockstep result.  No arithmetic changes.

Usage: python ref_gen.py --ref <reference root> --out <dir>
"""
from __future__ import annotations

import argparse
import os
import re
import sys

# (generated file, [(source file, kind, name)]); kinds: define, typedef, func
ITEMS = [
    ("uff.inc", [
        ("opencl/UFF.cl", "typedef", "cl_Mat3"),
        ("opencl/UFF.cl", "define", "float4Zero"),
        ("opencl/UFF.cl", "define", "float3Zero"),
        ("opencl/UFF.cl", "define", "EXCL_MAX"),
        ("opencl/UFF.cl", "define", "COULOMB_CONST"),
        ("opencl/UFF.cl", "func", "mixREQ_arithmetic"),       # UFF.cl:57-65
        ("opencl/UFF.cl", "func", "getLJQH"),                 # UFF.cl:82-95
        ("opencl/UFF.cl", "func", "modulo"),
        ("opencl/UFF.cl", "func", "make_inds_pbc"),           # UFF.cl:1384-1511: the sampler
        ("opencl/UFF.cl", "func", "choose_inds_pbc"),
        ("opencl/UFF.cl", "func", "basis"),
        ("opencl/UFF.cl", "func", "dbasis"),
        ("opencl/UFF.cl", "func", "fe1Dcomb"),
        ("opencl/UFF.cl", "func", "fe2d_comb"),
        ("opencl/UFF.cl", "func", "fe3d_pbc_comb"),
        ("opencl/UFF.cl", "func", "getNonBond_GridFF_Bspline"),      # UFF.cl:1524-1718
        ("opencl/UFF.cl", "func", "getNonBond_GridFF_Bspline_ex2"),  # UFF.cl:1722-
    ]),
    ("gridff.inc", [
        ("opencl/common.cl", "func", "modulo"),
        ("opencl/GridFF.cl", "func", "conv3x3_pbc"),
        ("opencl/gridff_build.cl", "func", "BsplineConv3D"),         # gridff_build.cl:8-61
        ("opencl/gridff_build.cl", "func", "make_MorseFF"),          # gridff_build.cl:217-347
    ]),
    ("surface.inc", [
        ("opencl/Surface.cl", "define", "COULOMB_CONST"),
        ("opencl/Surface.cl", "func", "cmul"),
        ("opencl/Surface.cl", "func", "compute_ewald_coefficients"),  # Surface.cl:716-767
        ("opencl/Surface.cl", "func", "eval_potential_full"),         # Surface.cl:834-906
        ("opencl/Surface.cl", "func", "eval_potential_brute"),        # Surface.cl:911-954
    ]),
]

# (function, text as in the reference, replacement): see the module docstring
PATCHES = [
    ("getNonBond_GridFF_Bspline_ex2",
     "        //barrier(CLK_LOCAL_MEM_FENCE);\n    }\n\n    } // insulate nbff",
     "        barrier(CLK_LOCAL_MEM_FENCE);\n    }\n\n    } // insulate nbff"),
]

VEC = r"(?:float|int|uint|double)[234]"


def skip_code(text, i, stop):
    """Index of the first character in `stop` at or after i, outside comments and literals."""
    n = len(text)
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            i = text.find("\n", i)
            i = n if i < 0 else i
            continue
        if text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
            continue
        if c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if c in stop:
            return i
        i += 1
    return -1


def match_close(text, i, open_c, close_c):
    """i at an opening bracket; index of its matching close, outside comments and literals."""
    depth = 0
    while True:
        i = skip_code(text, i, open_c + close_c)
        if i < 0:
            raise ValueError("unbalanced " + open_c + close_c)
        depth += 1 if text[i] == open_c else -1
        if depth == 0:
            return i
        i += 1


def line_of(text, i):
    return text.count("\n", 0, i) + 1


def comment_mask(text):
    """bytearray, 1 where text lies inside a comment or a string / char literal."""
    mask = bytearray(len(text))
    i, n = 0, len(text)
    while i < n:
        if text.startswith("//", i):
            k = text.find("\n", i)
            k = n if k < 0 else k
        elif text.startswith("/*", i):
            k = text.find("*/", i + 2)
            k = n if k < 0 else k + 2
        elif text[i] in "\"'":
            k = i + 1
            while k < n and text[k] != text[i]:
                k += 2 if text[k] == "\\" else 1
            k = min(k + 1, n)
        else:
            i += 1
            continue
        mask[i:k] = b"\x01" * (k - i)
        i = k
    return mask


def find_func(text, name):
    pat = re.compile(r"(?m)^[ \t]*((?:__kernel|inline|static|const|float|double|int|void|\w+)[\w \t\*]*?)\b"
                     + re.escape(name) + r"[ \t]*\(")
    mask = comment_mask(text)
    for m in pat.finditer(text):
        if mask[m.start() + len(m.group(0)) - len(m.group(0).lstrip())]:
            continue
        po = text.index("(", m.end() - 1)
        pc = match_close(text, po, "(", ")")
        k = pc + 1
        while k < len(text) and text[k] in " \t\r\n":
            k += 1
        if k < len(text) and text[k] == "{":
            end = match_close(text, k, "{", "}")
            start = text.rfind("\n", 0, m.start()) + 1
            return start, end + 1
    raise KeyError(name)


def find_define(text, name):
    m = re.search(r"(?m)^[ \t]*#define[ \t]+" + re.escape(name) + r"\b.*$", text)
    if not m:
        raise KeyError(name)
    return m.start(), m.end()


def find_typedef(text, name):
    m = re.search(r"}\s*" + re.escape(name) + r"\s*;", text)
    if not m:
        raise KeyError(name)
    start = text.rfind("typedef", 0, m.start())
    return start, m.end()


def translate(src):
    """OpenCL spellings -> the ref_cl.h spellings; arithmetic untouched."""
    src = re.sub(r"__attribute__\s*\(\(\s*reqd_work_group_size\s*\([^)]*\)\s*\)\)", "", src)
    src = re.sub(r"__local(\s+(?:const\s+)?\w+\s+\w+\s*\[)", r"static\1", src)
    out, i = [], 0
    mask = comment_mask(src)
    pat = re.compile(r"\(\s*(" + VEC + r")\s*\)\s*([({])")
    while True:
        m = pat.search(src, i)
        if not m:
            out.append(src[i:])
            break
        if mask[m.start()]:
            out.append(src[i:m.end()])
            i = m.end()
            continue
        out.append(src[i:m.start()])
        ty, br = m.group(1), m.group(2)
        o = m.end() - 1
        c = match_close(src, o, br, ")" if br == "(" else "}")
        inner = translate(src[o + 1:c])
        out.append(f"make_{ty}({inner})")
        i = c + 1
    return "".join(out)


def generate(ref, out_dir):
    os.makedirs(out_dir, exist_ok=True)
    cache = {}
    for fname, items in ITEMS:
        parts = [f"// generated by oracle/ref_gen.py from the reference's OpenCL sources; do not edit\n"]
        for path, kind, name in items:
            full = os.path.join(ref, path)
            if full not in cache:
                cache[full] = open(full, encoding="utf-8", errors="replace").read()
            text = cache[full]
            finder = {"func": find_func, "define": find_define, "typedef": find_typedef}[kind]
            a, b = finder(text, name)
            body = text[a:b]
            for fn, old, new in PATCHES:
                if fn == name:
                    if body.count(old) != 1:
                        raise ValueError(f"patch for {name} does not apply")
                    body = body.replace(old, new)
            parts.append(f'#line {line_of(text, a)} "{path}"\n{translate(body)}\n')
        with open(os.path.join(out_dir, fname), "w") as f:
            f.write("\n".join(parts))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SURFMOL_REFERENCE", ""), help="reference repository root")
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    if not a.ref or not os.path.isdir(os.path.join(a.ref, "opencl")):
        print("ref_gen.py: no reference tree (give --ref or SURFMOL_REFERENCE)", file=sys.stderr)
        return 2
    generate(a.ref, a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
