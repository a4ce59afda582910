"""Regenerate tests/golden/shipped_cases/ from the reference's case files.

The reference ships eleven BoltzTechs XML cases (MaterKit/BoltzTechs*.xml)
whose comments are GBK-encoded under an utf-8 declaration.  The fixtures are
those files with the comments and blank lines removed (the tags, values and
nesting unchanged), so the drop-in tests can read the shipped cases where the
reference tree is not present.

    python tests/golden/make_shipped_cases.py [/path/to/reference]
"""
from __future__ import annotations

import glob
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "shipped_cases")


def fixture_name(src: str) -> str:
    """'BoltzTechs - thermal.xml' -> 'boltztechs_thermal.xml'."""
    stem = os.path.splitext(os.path.basename(src))[0]
    return re.sub(r"[^a-z0-9]+", "_", stem.lower()).strip("_") + ".xml"


def strip(src: str) -> str:
    with open(src, "rb") as f:
        text = f.read().decode("latin-1")
    text = re.sub(r"<!--.*?-->", "", text, flags=re.S)
    lines = [ln.rstrip() for ln in text.splitlines()]
    body = "\n".join(ln for ln in lines if ln.strip())
    return body.encode("latin-1").decode("ascii") + "\n"


def main(ref: str) -> None:
    files = sorted(glob.glob(os.path.join(ref, "MaterKit", "BoltzTechs*.xml")))
    if not files:
        raise SystemExit(f"no BoltzTechs*.xml under {ref}/MaterKit")
    os.makedirs(OUT, exist_ok=True)
    for src in files:
        with open(os.path.join(OUT, fixture_name(src)), "w") as f:
            f.write(strip(src))
        print(os.path.basename(src), "->", fixture_name(src))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
