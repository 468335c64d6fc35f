"""Regenerate ``it1992.json`` from the reference's form-factor table.

The reference evaluates atomic form factors from a 9-coefficient table
(a1..a4, b1..b4, c; International Tables for Crystallography, 1992) held in
``cpp-src/Utilities/Scattering.cpp:9-189``.  Parity of I(q) requires the very
same coefficients, so this script parses that table as text and writes it as
JSON; it is run once, by hand, where the reference sources are available:

    python pycusaxs_b200/data/extract_form_factors.py <reference-root>

The JSON maps element symbol -> [a1, a2, a3, a4, b1, b2, b3, b4, c] and keeps
the reference's key order.  Values are kept as the decimal strings of the
source and parsed to float32 by the loader, exactly as the reference's
``std::vector<float>`` initialiser does.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

_ENTRY = re.compile(
    r'\{\s*"([^"]+)"\s*,\s*\{\s*\{([^}]*)\}\s*,\s*(?:/\*.*?\*/\s*)?\{([^}]*)\}\s*,\s*\{([^}]*)\}\s*\}\s*\}',
    re.S,
)


def parse(text: str) -> dict[str, list[str]]:
    start = text.index("it1992")
    body = text[start:]
    out: dict[str, list[str]] = {}
    for m in _ENTRY.finditer(body):
        name = m.group(1)
        a = [v.strip() for v in m.group(2).split(",") if v.strip()]
        b = [v.strip() for v in m.group(3).split(",") if v.strip()]
        c = [v.strip() for v in m.group(4).split(",") if v.strip()]
        if len(a) != 4 or len(b) != 4 or len(c) != 1:
            raise ValueError(f"malformed entry for {name!r}: {a} {b} {c}")
        out[name] = a + b + c
    return out


def main(argv: list[str]) -> int:
    if len(argv) < 2:
        print("usage: extract_form_factors.py <reference-root>", file=sys.stderr)
        return 2
    root = Path(argv[1])
    src = root / "cpp-src" / "Utilities" / "Scattering.cpp"
    table = parse(src.read_text())
    dest = Path(__file__).with_name("it1992.json")
    lines = [f"{json.dumps(k)}: {json.dumps(v)}" for k, v in table.items()]
    dest.write_text("{\n" + ",\n".join(lines) + "\n}\n")
    print(f"wrote {len(table)} elements to {dest}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main(sys.argv))
