"""Generate mc_tables.h from the reference's marching-cells tables.

The dual marching cells step must use exactly the reference's corner
reordering and triangulation tables (the public-domain Paul Bourke tables that
DualMarchingCellTables.cpp:17-314 carries), otherwise case codes and triangle
lists could not match.  This script reads that file from a checkout of the
reference, checks the edge-cuttings table against the one derived from the
corner signs, and writes the packed header this package compiles against.

Usage: python gen_mc_tables.py <path to DualMarchingCellTables.cpp>
"""
import re
import sys
from pathlib import Path


def _block(src, name):
    m = re.search(name + r"[^=]*=\s*\{(.*?)\};", src, re.S)
    if not m:
        raise SystemExit("table %s not found" % name)
    body = re.sub(r"//[^\n]*", "", m.group(1))
    return [int(v, 0) for v in re.findall(r"-?0x[0-9a-fA-F]+|-?\d+", body)]


def main(path):
    src = Path(path).read_text()
    reorder = _block(src, "MC_CORNER_REORDERING")
    cuts = _block(src, "MC_EDGE_CUTTINGS_TABLE")
    ends = _block(src, "MC_EDGE_ENDS")
    tris = _block(src, "MC_TRIANGULATION_TABLE")
    assert len(reorder) == 8 and len(cuts) == 256 and len(ends) == 24 and len(tris) == 256 * 16
    ends2 = [ends[2 * i:2 * i + 2] for i in range(12)]
    for code in range(256):
        derived = 0
        for e, (a, b) in enumerate(ends2):
            if ((code >> a) ^ (code >> b)) & 1:
                derived |= 1 << e
        assert derived == cuts[code], code
    rows = []
    for code in range(256):
        row = tris[16 * code:16 * code + 16]
        rows.append("{" + ",".join(str(v) for v in row) + "}")
    out = []
    out.append("/* Generated by gen_mc_tables.py from the reference's")
    out.append(" * DualMarchingCellTables.cpp (public-domain Paul Bourke marching cubes")
    out.append(" * tables).  Do not edit by hand. */")
    out.append("#ifndef TSR_MC_TABLES_H")
    out.append("#define TSR_MC_TABLES_H")
    out.append("#include <stdint.h>")
    out.append("#define TSR_MC_CORNER_REORDERING_INIT {" + ",".join(map(str, reorder)) + "}")
    out.append("#define TSR_MC_EDGE_ENDS_INIT {" + ",".join("{%d,%d}" % tuple(e) for e in ends2) + "}")
    out.append("#define TSR_MC_TRIANGLES_INIT { \\")
    for i, r in enumerate(rows):
        out.append("  " + r + ("," if i < 255 else "") + " \\")
    out.append("}")
    out.append("static const uint8_t MC_CORNER_REORDERING[8] = TSR_MC_CORNER_REORDERING_INIT;")
    out.append("static const uint8_t MC_EDGE_ENDS[12][2] = TSR_MC_EDGE_ENDS_INIT;")
    out.append("static const int8_t MC_TRIANGLES[256][16] = TSR_MC_TRIANGLES_INIT;")
    out.append("static inline const int8_t *mc_triangles(uint32_t code) { return MC_TRIANGLES[code]; }")
    out.append("#endif")
    dst = Path(__file__).with_name("mc_tables.h")
    dst.write_text("\n".join(out) + "\n")
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1])
