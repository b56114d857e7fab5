#!/usr/bin/env python3
"""Count the arithmetic of the reference's point integrands (test infrastructure).

phys/ge/residual.c and phys/ge/tangent.c are machine-generated straight-line C:
one assignment per temporary or output, operands written as *(u+N), *(e+N),
*(par+N).  This script counts, per call, the binary additions / subtractions,
multiplications, divisions and pow() calls on the right-hand sides (pow counted
as one operation; a leading unary minus is not counted).  The result pins the
integrand term of the residual's algorithmic flop count that bench.py uses.

Usage: python oracle/count_integrand_flops.py [REFERENCE_DIR]
(default: $IGAP4_REFERENCE, else a directory named "reference" beside this
repository).  Prints one line per file.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_dir(argv):
    if len(argv) > 1:
        return argv[1]
    return os.environ.get("IGAP4_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def count(path):
    src = open(path).read()
    body = src[src.index("{") + 1:]
    body = re.sub(r"\*\((\w+)\+(\d+)\)", "V", body)
    body = re.sub(r"\*\((\w+)\)", "V", body)
    add = mul = div = pw = 0
    for stmt in body.split(";"):
        if "=" not in stmt:
            continue
        rhs = stmt.split("=", 1)[1]
        pw += len(re.findall(r"pow\(", rhs))
        rhs = re.sub(r"(^|[\(,=])\s*-", r"\1", rhs.replace("pow(", "P("))
        add += len(re.findall(r"[+-]", rhs))
        mul += rhs.count("*")
        div += rhs.count("/")
    return add, mul, div, pw


def main(argv):
    ref = reference_dir(argv)
    for rel in ("phys/ge/residual.c", "phys/ge/tangent.c"):
        path = os.path.join(ref, rel)
        if not os.path.exists(path):
            print("%s: not found under %s" % (rel, ref))
            return 1
        a, m, d, p = count(path)
        print("%s: %d add/sub, %d mul, %d div, %d pow = %d operations per call" % (rel, a, m, d, p, a + m + d + p))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
