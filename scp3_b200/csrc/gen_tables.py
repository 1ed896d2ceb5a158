"""Regenerate the two constant-data headers that must match the reference bit for bit.

* ``sobol_dirnum.h``: the primitive-polynomial codes and the initial direction
  numbers of the 62-bit Sobol generator, dimensions 1..1111.  They are the data
  that ``i8_sobol`` fills in before its Bratley-Fox recurrence
  (sobol.cpp:14308-14420 ``poly[]``, sobol.cpp:14440-27670 ``v[i][j] = ...``).
  The recurrence itself is restated in our own code (``tables.cpp``).
* ``ps_coeffs.h``: the Partridge-Schwenke monomer expansion (245 terms, four
  coefficient sets combined at start-up, ps.cpp:18-458) and the 84-term dipole
  moment surface (ps.cpp:417-466) used by TTM3-F.

Both tables are published physical / number-theoretic data; a Sobol sequence or
a potential with different numbers is a different sequence or potential, so the
numbers are kept exactly as the reference writes them (the decimal literals are
re-emitted verbatim so the compiler parses identical doubles).

Usage (only where the reference tree is present; its root is the argument, or
$SCP3_REFERENCE when no argument is given):
    python scp3_b200/csrc/gen_tables.py <reference tree>
"""
import os
import re
import sys


def _i8_sobol_span(lines):
    start = next(i for i, l in enumerate(lines) if l.startswith("void i8_sobol ("))
    end = next(i for i in range(start, len(lines)) if lines[i].startswith("double *i8_sobol_generate"))
    return lines[start:end]


def sobol_tables(src):
    lines = open(src).read().splitlines()
    body = _i8_sobol_span(lines)
    text = "\n".join(body)
    m = re.search(r"static long long int poly\[DIM_MAX2\]\s*=\s*\{([^}]*)\}", text)
    poly = [int(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]
    assert len(poly) == 1111, len(poly)
    init = {}
    for l in body:
        mm = re.match(r"\s*v\[\s*(\d+)\]\[\s*(\d+)\]\s*=\s*(\d+)\s*;", l)
        if mm:
            init[(int(mm.group(1)), int(mm.group(2)))] = int(mm.group(3))
    maxj = max(j for _, j in init) + 1
    table = [[init.get((i, j), 0) for j in range(maxj)] for i in range(1111)]
    # every row i>=1 must have exactly deg(poly[i]) initial values
    for i in range(1, 1111):
        deg = poly[i].bit_length() - 1
        for j in range(deg):
            assert (i, j) in init, (i, j)
    return poly, table, maxj


def ps_tables(src):
    text = open(src).read()

    def arr(name, kind):
        m = re.search(r"const (?:double|size_t) %s\[(\d+)\]\s*=\s*\{([^}]*)\}" % name, text)
        n = int(m.group(1))
        vals = [x.strip() for x in m.group(2).replace("\n", " ").split(",") if x.strip()]
        assert len(vals) == n, (name, len(vals), n)
        if kind == "int":
            vals = [str(int(v)) for v in vals]
        return vals

    out = {}
    for name in ("c5zA", "cbasis", "ccore", "crest", "coefD"):
        out[name] = arr(name, "double")
    for name in ("idx1", "idx2", "idx3", "idxD0", "idxD1", "idxD2"):
        out[name] = arr(name, "int")
    return out


def emit_c_array(f, ctype, name, vals, per_line=6):
    f.write("static const %s %s[%d] = {\n" % (ctype, name, len(vals)))
    for k in range(0, len(vals), per_line):
        f.write("    " + ", ".join(vals[k:k + per_line]) + ",\n")
    f.write("};\n\n")


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    poly, table, maxj = sobol_tables(os.path.join(ref, "sobol.cpp"))
    with open(os.path.join(here, "sobol_dirnum.h"), "w") as f:
        f.write("/* Generated by gen_tables.py from the reference's i8_sobol data\n"
                " * (sobol.cpp:14308-14420 poly[], sobol.cpp:14440-27670 initial v[i][j]).\n"
                " * Do not edit: published Sobol direction-number data, kept identical so that\n"
                " * the point sequence is the reference's. */\n")
        f.write("#pragma once\n#include <stdint.h>\n\n")
        f.write("#define SCP3_SOBOL_MAX_DIMS 1111\n#define SCP3_SOBOL_INIT_COLS %d\n\n" % maxj)
        emit_c_array(f, "uint16_t", "scp3_sobol_poly", [str(p) for p in poly], 12)
        f.write("static const uint16_t scp3_sobol_vinit[1111][%d] = {\n" % maxj)
        for row in table:
            f.write("    {" + ", ".join(str(v) for v in row) + "},\n")
        f.write("};\n")
    ps = ps_tables(os.path.join(ref, "ps.cpp"))
    with open(os.path.join(here, "ps_coeffs.h"), "w") as f:
        f.write("/* Generated by gen_tables.py from the reference's Partridge-Schwenke data\n"
                " * (ps.cpp:18-458: monomer expansion c5zA/cbasis/ccore/crest and exponent\n"
                " * indices idx1..3; ps.cpp:417-466: dipole-moment surface coefD, idxD0..2).\n"
                " * Do not edit: published potential parameters kept identical. */\n")
        f.write("#pragma once\n\n")
        for name in ("c5zA", "cbasis", "ccore", "crest"):
            emit_c_array(f, "double", "scp3_ps_" + name, ps[name], 3)
        for name in ("idx1", "idx2", "idx3"):
            emit_c_array(f, "unsigned char", "scp3_ps_" + name, ps[name], 20)
        emit_c_array(f, "double", "scp3_ps_coefD", ps["coefD"], 3)
        for name in ("idxD0", "idxD1", "idxD2"):
            emit_c_array(f, "unsigned char", "scp3_ps_" + name, ps[name], 20)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SCP3_REFERENCE")
    if not ref:
        sys.exit("usage: gen_tables.py <reference tree>  (or set SCP3_REFERENCE)")
    main(ref)
