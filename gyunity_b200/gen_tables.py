"""Generate the Sobol' tables header from the reference's table sources.

The Sobol' generator matrices (Joe-Kuo direction numbers as tabulated by
Gruenschloss 2012, reference ``sampler/Sobol.cpp:38``) and the per-pixel
enumeration matrices (``sampler/SobolEnum.cpp:5`` and ``:709``) are data of
the reference. They are not copied into this repository: this script reads
them from a reference checkout and writes ``gyunity_b200/_gen/sobol_tables.h``
(git-ignored). The built libraries embed the tables, so machines without the
reference checkout only need the built ``.so`` files.

Layout of the generated header:
  GYT_SOBOL_DIMS = 1024, GYT_SOBOL_COLS = 52
  static const uint32_t gyt_sobol_matrices[1024 * 52];
  GYT_ENUM_M = number of enumeration levels (max log2 resolution)
  static const uint64_t gyt_vdc_sobol[GYT_ENUM_M][52];
  static const uint64_t gyt_vdc_sobol_inv[GYT_ENUM_M][52];
"""
import hashlib
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_gen")
OUT = os.path.join(OUT_DIR, "sobol_tables.h")
HEX = re.compile(r"0x[0-9a-fA-F]+")


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _sobol_matrices(path):
    text = _strip_comments(open(path).read())
    start = text.index("Matrices::matrices[")
    body = text[text.index("{", start) + 1:text.index("};", start)]
    vals = [int(h, 16) for h in HEX.findall(body)]
    if len(vals) != 1024 * 52:
        raise RuntimeError("unexpected Sobol matrix count %d" % len(vals))
    return vals


def _jagged(text, name):
    start = text.index(name)
    i = text.index("{", start) + 1
    rows, depth, cur = [], 0, None
    while True:
        ch = text[i]
        if ch == "{":
            depth += 1
            cur = i + 1
        elif ch == "}":
            if depth == 0:
                break
            depth -= 1
            rows.append([int(h, 16) for h in HEX.findall(text[cur:i])])
        i += 1
    return rows


def _enum_tables(path):
    text = _strip_comments(open(path).read())
    fwd = _jagged(text, "vdc_sobol_matrices[]")
    inv = _jagged(text, "vdc_sobol_matrices_inv[]")
    # the inverse table carries one more level than the forward one; only
    # levels present in both are usable (m = log2 of the padded resolution)
    n = min(len(fwd), len(inv))
    fwd, inv = fwd[:n], inv[:n]
    for r in fwd + inv:
        if len(r) > 52:
            raise RuntimeError("enumeration row longer than 52 columns")
    return fwd, inv


def generate(reference=None, force=False):
    """Writes the generated header from the reference checkout at
    ``reference`` (else $GYUNITY_REFERENCE); without a checkout an existing
    header is kept."""
    reference = reference or os.environ.get("GYUNITY_REFERENCE")
    src = os.path.join(reference, "Gyunity", "src", "sampler") if reference else None
    if not src or not os.path.isdir(src):
        if os.path.exists(OUT):
            return OUT
        raise FileNotFoundError("Sobol tables: no generated header and no reference checkout (pass its location or "
                                "set GYUNITY_REFERENCE); looked at %r" % reference)
    if os.path.exists(OUT) and not force:
        return OUT
    mats = _sobol_matrices(os.path.join(src, "Sobol.cpp"))
    fwd, inv = _enum_tables(os.path.join(src, "SobolEnum.cpp"))
    os.makedirs(OUT_DIR, exist_ok=True)
    lines = ["// Generated by gyunity_b200/gen_tables.py from the reference's Sobol' tables. Do not edit.",
             "#pragma once", "#include <stdint.h>",
             "#define GYT_SOBOL_DIMS 1024", "#define GYT_SOBOL_COLS 52", "#define GYT_ENUM_M %d" % len(fwd),
             "static const uint32_t gyt_sobol_matrices[GYT_SOBOL_DIMS * GYT_SOBOL_COLS] = {"]
    for k in range(0, len(mats), 8):
        lines.append("  " + ", ".join("0x%08xu" % v for v in mats[k:k + 8]) + ",")
    lines.append("};")
    for nm, tab in (("gyt_vdc_sobol", fwd), ("gyt_vdc_sobol_inv", inv)):
        lines.append("static const uint64_t %s[GYT_ENUM_M][52] = {" % nm)
        for row in tab:
            row = row + [0] * (52 - len(row))
            lines.append("  {" + ", ".join("0x%xull" % v for v in row) + "},")
        lines.append("};")
    data = "\n".join(lines) + "\n"
    digest = hashlib.sha256(data.encode()).hexdigest()[:16]
    data += "#define GYT_TABLES_DIGEST \"%s\"\n" % digest
    with open(OUT, "w") as f:
        f.write(data)
    return OUT


if __name__ == "__main__":
    print(generate(sys.argv[1] if len(sys.argv) > 1 else None, force=True))
