"""Extract the Johnson & Christy (Phys. Rev. B 6, 4370, 1972) gold table.

The reference ships the published (wavelength/um, n, k) rows of the gold
dataset inside crates/lumina-materials/src/johnson_christy.rs (the
`gold()` constructor, lines 51-97).  This script reads those rows as text and
writes them to ``johnson_christy_au.csv`` next to this file, so the package
carries the data without reading the reference at run time.

Usage: python extract_jc_table.py <path of the Lumina source tree>
"""
import os
import re
import sys


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "crates/lumina-materials/src/johnson_christy.rs")
    text = open(src).read()
    start = text.index("pub fn gold()")
    end = text.index("pub fn silver()")
    body = text[start:end]
    rows = re.findall(r"\(\s*([0-9.]+)\s*,\s*([0-9.]+)\s*,\s*([0-9.]+)\s*\)", body)
    if len(rows) < 10:
        raise SystemExit("gold table not found")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "johnson_christy_au.csv")
    with open(out, "w") as f:
        f.write("# Johnson & Christy 1972, gold: wavelength_um,n,k\n")
        for wl, n, k in rows:
            f.write(f"{wl},{n},{k}\n")
    print(f"wrote {len(rows)} rows to {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
