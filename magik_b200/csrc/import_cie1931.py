#!/usr/bin/env python
"""One-off import of the CIE 1931 2-degree standard colorimetric observer.

    python magik_b200/csrc/import_cie1931.py /root/reference

Writes `cie1931_2deg.inc` beside this file: the colour-matching functions
x(l), y(l), z(l) at 1 nm from 360 to 830 nm (471 rows), the published CIE
standard data (CIE 015 / ISO/CIE 11664-1).  The values are read from the
reference's own tabulation (src/renderer/color/color_matching_functions.cuh,
`generic_color_matching_function_t<MAGIK_CMF_CIE_1931>::values`) so that the
library integrates exactly the numbers the reference integrates; the
generated file is committed and the build never runs this script.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "cie1931_2deg.inc")


def read_table(ref_root):
    path = os.path.join(ref_root, "src", "renderer", "color", "color_matching_functions.cuh")
    text = open(path).read()
    body = text[text.index("values[n_entries]"):]
    body = body[body.index("{") + 1:body.index("};")]
    rows = re.findall(r"\{\s*([-+0-9.eE]+)f?\s*,\s*([-+0-9.eE]+)f?\s*,\s*([-+0-9.eE]+)f?\s*\}", body)
    if len(rows) != 471:
        raise SystemExit(f"expected 471 rows, found {len(rows)}")
    return rows


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    rows = read_table(ref_root)
    with open(OUT, "w") as f:
        f.write("// CIE 1931 2-degree standard colorimetric observer (CIE 015, ISO/CIE 11664-1):\n")
        f.write("// x(l), y(l), z(l) at l = 360, 361, ..., 830 nm.  Generated by import_cie1931.py.\n")
        for i, (x, y, z) in enumerate(rows):
            f.write(f"{{{x}f, {y}f, {z}f}},  // {360 + i}\n")
    print(f"wrote {OUT}: {len(rows)} rows")


if __name__ == "__main__":
    main()
