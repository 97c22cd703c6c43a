#!/usr/bin/env python
"""Copies the code blocks of INTEGRATION.md marked `<!-- compiled: NAME -->`
into OUT/integration_NAME.inc, unchanged, for the integration adapter
(oracle/ref/integration_adapter.cpp) to compile (test infrastructure only).

usage: extract_snippets.py INTEGRATION.md OUT_DIR
"""
import os
import re
import sys

MARK = re.compile(r"<!-- compiled: ([a-z0-9_]+) -->\s*\n```cpp\n(.*?)\n```", re.S)


def snippets(text):
    """{name: code} of the marked blocks, in file order."""
    out = {}
    for m in MARK.finditer(text):
        if m.group(1) in out:
            raise ValueError(f"snippet {m.group(1)} marked twice")
        out[m.group(1)] = m.group(2) + "\n"
    return out


def main(src, out_dir):
    os.makedirs(out_dir, exist_ok=True)
    for name, code in snippets(open(src).read()).items():
        path = os.path.join(out_dir, f"integration_{name}.inc")
        # rewrite only on change, so that make sees stable timestamps
        if not os.path.exists(path) or open(path).read() != code:
            with open(path, "w") as f:
                f.write(code)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
