"""TEST INFRASTRUCTURE ONLY.  Writes oracle/_ref/ref_stein.cpp: a thin harness
that compiles the reference's gradient-estimator formulas (TripleExcitations.h,
included unchanged inside a class that supplies the members it reads: q, Vq
with colptr(k), V with n_rows and operator[]) and exposes each formula by index
through extern "C" functions, so the oracle's restatement can be pinned formula
by formula.

    python3 oracle/gen_ref_stein.py <reference dir> <output .cpp>
"""
import re
import sys


def main(ref, out):
    src = open(ref + "/TripleExcitations.h").read()
    sigs = []
    for m in re.finditer(r"^double\s+(\w+)\(([^)]*)\)", src, re.M):
        name, params = m.group(1), [p.split()[-1] for p in m.group(2).split(",") if p.strip()]
        if name not in [s[0] for s in sigs]:
            sigs.append((name, params))
    lines = [
        "// generated by oracle/gen_ref_stein.py -- test infrastructure only",
        "#include <cmath>",
        "#include <cstddef>",
        "#define __assume_aligned(x, n)",
        "using std::sqrt;",
        "static inline double square(double x) { return x * x; }   // arma::square on a scalar",
        "namespace {",
        "struct MatView { double* base; int rows; double* colptr(int k) const { return base + (std::size_t)k * rows; } };",
        "struct VecView { double* base; int n_rows; double& operator[](int i) const { return base[i]; } };",
        "struct RefStein {",
        "    MatView q, Vq;",
        "    VecView V;",
        '#include "TripleExcitations.h"',
        "};",
        "const char* kNames[] = {%s};" % ", ".join('"%s"' % s[0] for s in sigs),
        "const char* kParams[] = {%s};" % ", ".join('"%s"' % ",".join(s[1]) for s in sigs),
        "}  // namespace",
        'extern "C" int ref_stein_count() { return %d; }' % len(sigs),
        'extern "C" const char* ref_stein_name(int i) { return kNames[i]; }',
        'extern "C" const char* ref_stein_params(int i) { return kParams[i]; }',
        "// q, Vq: [mode][sample] (sample-contiguous, the reference's transposed layout); V: [sample]",
        'extern "C" double ref_stein_eval(int i, double* q, double* V, double* Vq, int n, const int* a)',
        "{",
        "    RefStein r{MatView{q, n}, MatView{Vq, n}, VecView{V, n}};",
        "    switch (i) {",
    ]
    for i, (name, params) in enumerate(sigs):
        args = ", ".join("a[%d]" % k for k in range(len(params)))
        lines.append("        case %d: return r.%s(%s);" % (i, name, args))
    lines += ["    }", "    return 0.0;", "}", ""]
    open(out, "w").write("\n".join(lines))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
