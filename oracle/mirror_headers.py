"""Write an access-opened mirror of the reference headers (oracle build step).

Usage: python3 mirror_headers.py <reference root> <output dir>

Copies every header under <ref>/mdtk and <ref>/yaatk into <out>, keeping the
directory structure, with `private:`/`protected:` labels turned into
`public:` and a `public:` label inserted after each class-opening brace.  The
oracle harness compiles against the mirror so it can read spline tables and
parameters the reference keeps private (e.g. mdtk/potentials/manybody/AIREBO/
cubici.hpp:112-204, AIREBO_LJ.hpp:128-134).  Output goes to the oracle's build
folder only; it is never committed.
"""
import os
import re
import sys

ACCESS = re.compile(r"\b(private|protected)\s*:(?!:)")
CLASS_OPEN = re.compile(r"(\bclass\s+\w+[^;{()]*\{)")


def mirror(src_root: str, out_root: str) -> int:
    n = 0
    for top in ("mdtk", "yaatk"):
        for dirpath, _, files in os.walk(os.path.join(src_root, top)):
            for name in files:
                if not name.endswith((".hpp", ".h", ".inc")):
                    continue
                src = os.path.join(dirpath, name)
                rel = os.path.relpath(src, src_root)
                dst = os.path.join(out_root, rel)
                os.makedirs(os.path.dirname(dst), exist_ok=True)
                with open(src, "r", encoding="latin-1") as f:
                    text = f.read()
                text = ACCESS.sub("public:", text)
                text = CLASS_OPEN.sub(r"\1 public:", text)
                with open(dst, "w", encoding="latin-1") as f:
                    f.write(text)
                n += 1
    return n


if __name__ == "__main__":
    count = mirror(sys.argv[1], sys.argv[2])
    print(f"mirrored {count} headers into {sys.argv[2]}")
