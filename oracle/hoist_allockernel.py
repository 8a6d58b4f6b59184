#!/usr/bin/env python3
"""Generate the "allocKernel hoisted" variant of the reference's kernel.c (test infrastructure).

The reference's driver loop processAntennasAndBaselinePara (kernel.c:709-827) declares an
FxKernel and calls allocKernel for every (FFT, antenna) pair (kernel.c:727-728): allocKernel
builds the same geometry tables and IPP FFT spec every time and never frees them.  This
script writes a copy of kernel.c, into the build directory only, in which that declaration and
call sit once before the FFT loop of that function.  allocKernel depends only on the geometry
(kernel.c:117-187), so the copy computes exactly what the original computes, without the
per-(FFT, antenna) rebuild and leak.  It is the secondary CPU figure next to the as-written one.

    python3 hoist_allockernel.py <reference kernel.c> <output .c>

Exits non-zero, writing nothing, unless the two lines occur exactly once inside
processAntennasAndBaselinePara, after its local declarations.
"""
import re
import sys


def hoist(src: str) -> str:
    fn = src.index("void processAntennasAndBaselinePara(")
    body = src.index("{", fn)
    end = src.index("\nvoid processBaselinePara(", body)
    part = src[body:end]
    decl = re.compile(r"\n[ \t]*FxKernel kernel;\n[ \t]*allocKernel\(&kernel,[^;]*\);")
    m = list(decl.finditer(part))
    if len(m) != 1:
        raise SystemExit(f"expected one FxKernel declaration + allocKernel call in the driver loop, found {len(m)}")
    call = m[0].group(0)
    part = part[:m[0].start()] + part[m[0].end():]
    anchor = "int netdelaysamples, offset;"
    if part.count(anchor) != 1:
        raise SystemExit("local declaration anchor not found once")
    part = part.replace(anchor, anchor + "\n    /* hoisted out of the FFT x antenna loop */" + call, 1)
    return src[:body] + part + src[end:]


def main(argv):
    if len(argv) != 3:
        raise SystemExit(__doc__)
    with open(argv[1]) as f:
        out = hoist(f.read())
    with open(argv[2], "w") as f:
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
