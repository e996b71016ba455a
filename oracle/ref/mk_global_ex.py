"""Write the extern-declaration companion of the reference's src/global.h.

FARGO3D's build derives global_ex.h from global.h by turning every
declaration line into an ``extern`` declaration (initialisers dropped).  This
script applies that same rule so that the reference's hot-path sources can be
compiled outside its build system.  Usage: mk_global_ex.py <global.h> <out>.
"""
import re
import sys

src, out = sys.argv[1], sys.argv[2]
lines = []
with open(src) as fh:
    for line in fh.read().splitlines():
        m = re.match(r"([^/=]*)[=|;]", line)
        lines.append("extern " + m.group(1).strip() + ";" if m else line)
with open(out, "w") as fh:
    fh.write("\n".join(lines) + "\n")
