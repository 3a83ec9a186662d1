"""Writes blackbody_table.h: the reference's temperature -> RGB table.

The reference colours stars from a 391-entry blackbody table (1000 K to
40000 K in 100 K steps, RGB triplets; annemiekie/BlackTracer BT/Const.h:7,
the same values as BT/kernel.cuh:45).  The star colours of this build must
match the reference's bit for bit, so the table is the same data; this
script reads it from the reference tree once and writes the header, which is
committed.

    python blacktracer_b200/csrc/make_blackbody_table.py [reference tree]

The tree defaults to $BT_REFERENCE_DIR.
"""
import os
import re
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BT_REFERENCE_DIR", "")
if not ref:
    sys.exit("usage: make_blackbody_table.py <reference tree> (or set BT_REFERENCE_DIR)")
src = open(os.path.join(ref, "BlackTracer2", "BlackTracer", "Const.h")).read()
body = src[src.index("tempToRGBx"):]
body = body[body.index("{") + 1: body.index("}")]
vals = [int(v) for v in re.findall(r"-?\d+", body)]
assert len(vals) == 1173, len(vals)
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "blackbody_table.h")
with open(out, "w") as f:
    f.write("// blackbody_table.h -- generated by make_blackbody_table.py; do not edit.\n")
    f.write("// Blackbody temperature -> RGB (1000 K .. 40000 K, 100 K steps), 391 RGB\n")
    f.write("// triplets: the data of the reference's table (BT/Const.h:7,\n")
    f.write("// BT/kernel.cuh:45), needed bit for bit for colour parity.\n")
    f.write("#pragma once\n\n#define BT_BLACKBODY_RGB_VALUES \\\n")
    for k in range(0, 1173, 18):
        f.write("    " + ", ".join(str(v) for v in vals[k:k + 18]) + ", \\\n")
    f.write("\n\nnamespace bt {\n\nconstexpr int kBlackbodyEntries = 391;\n")
    f.write("__constant__ const int kBlackbodyRGB[1173] = {BT_BLACKBODY_RGB_VALUES};\n")
    f.write("static const int kBlackbodyRGBHost[1173] = {BT_BLACKBODY_RGB_VALUES};\n\n")
    f.write("__host__ __device__ __forceinline__ int blackbody(int k) {\n")
    f.write("#ifdef __CUDA_ARCH__\n  return kBlackbodyRGB[k];\n#else\n")
    f.write("  return kBlackbodyRGBHost[k];\n#endif\n}\n\n}  // namespace bt\n")
print(out)
