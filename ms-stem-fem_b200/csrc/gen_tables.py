#!/usr/bin/env python3
"""Regenerate the two data tables that must equal the reference's exactly.

Run from the repository root with the reference sources present:

    python ms-stem-fem_b200/csrc/gen_tables.py /path/to/ms-stem-fem

1. ``kirkland_table.inc`` -- the 12 Kirkland fit parameters for Z = 1..103
   exactly as the reference stores them in ``scatterer_param_LUT.hpp:119-1561``
   (including the field ordering that file's comment at ``:96-117`` calls
   mistaken; parity needs the table as stored, not as published).  The
   decimal literals are kept verbatim so they parse to the same doubles.
2. ``mass_table.inc`` -- the atomic-mass -> Z rules of ``guessZ``
   (``tem_io.cpp:1030-1258``), one row per rule in the order they are tried:
   an optional exact mass, an inclusive lower bound, an upper bound and
   whether that upper bound is inclusive.

Only the numbers are taken; the layout of both tables is this project's own.
"""
import re
import sys
from pathlib import Path


def kirkland(src: Path) -> str:
    text = (src / "scatterer_param_LUT.hpp").read_text()
    pat = re.compile(
        r"^\s*\(get_paramPtr\(\s*(\d+)\s*\)\)->([abcd])\[(\d)\]\s*=\s*([-+0-9.eE]+)\s*;",
        re.M)
    table = {}
    for z, field, k, val in pat.findall(text):
        table[(int(z), field, int(k))] = val
    rows = []
    for z in range(1, 104):
        vals = [table[(z, f, k)] for f in "abcd" for k in range(3)]
        rows.append("  /* Z=%3d */ {%s}," % (z, ", ".join(vals)))
    return ("/* Generated by gen_tables.py from the reference's parameter table.\n"
            " * Row Z-1 holds {a0,a1,a2, b0,b1,b2, c0,c1,c2, d0,d1,d2} as stored. */\n"
            + "\n".join(rows) + "\n")


def mass_rules(src: Path) -> str:
    lines = (src / "tem_io.cpp").read_text().splitlines()
    start = next(i for i, l in enumerate(lines) if "TEM_NS::guessZ" in l)
    body = []
    for l in lines[start:]:
        body.append(l.split("//")[0])
        if l.strip() == "}" and len(body) > 5:
            break
    joined = " ".join(body)
    rows = []
    for clause, z in re.findall(r"if\s*(.*?)ZZ\s*=\s*(\d+)\s*;", joined):
        exact = re.findall(r"mass\s*==\s*([0-9.]+)", clause)
        lo = re.findall(r"mass\s*>=\s*([0-9.]+)", clause)
        hi_inc = re.findall(r"mass\s*<=\s*([0-9.]+)", clause)
        hi_exc = re.findall(r"mass\s*<\s*([0-9.]+)", clause)
        assert len(lo) == 1 and len(hi_inc) + len(hi_exc) == 1, clause
        hi, inclusive = (hi_inc[0], 1) if hi_inc else (hi_exc[0], 0)
        ex = exact[0] if exact else "-1.0"
        rows.append("  {%s, %s, %s, %d, %s}," % (ex, lo[0], hi, inclusive, z))
    return ("/* Generated by gen_tables.py from the reference's mass -> Z rules.\n"
            " * {exact mass or -1, lower (inclusive), upper, upper inclusive, Z},\n"
            " * tried in order; the first match wins. */\n"
            + "\n".join(rows) + "\n")


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: gen_tables.py <path of the reference ms-stem-fem checkout>")
    ref = Path(sys.argv[1])
    src = ref / "src"
    here = Path(__file__).resolve().parent
    (here / "kirkland_table.inc").write_text(kirkland(src))
    (here / "mass_table.inc").write_text(mass_rules(src))


if __name__ == "__main__":
    main()
