"""INTEGRATION.md's marked code blocks are what the integration adapter
compiles (CPU checks; the runs on a GPU are in test_integration_snippets_gpu).

oracle/ref/extract_snippets.py copies each block marked
`<!-- compiled: NAME -->` into oracle/_ref/integration_NAME.inc, and
oracle/ref/integration_adapter.cpp includes them, compiled against the
reference's headers (make -C oracle integ)."""
import os
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))

pytestmark = pytest.mark.skipif(not oracle.integ_available(), reason="adapter not built")


def test_marked_blocks_are_the_compiled_ones():
    import extract_snippets

    blocks = extract_snippets.snippets(open(os.path.join(ROOT, "INTEGRATION.md")).read())
    assert set(blocks) == {"header", "mcf_u16", "mcf_f32", "pressure", "splat", "g2p_mr"}
    for name, code in blocks.items():
        path = os.path.join(oracle.OUT, f"integration_{name}.inc")
        assert open(path).read() == code, f"{path} is older than INTEGRATION.md"


def test_adapter_exports_the_snippet_runners():
    L = oracle.integ()
    for sym in ("integ_mcf_u16", "integ_mcf_f32", "integ_pressure", "integ_splat",
                "integ_g2p_mr"):
        assert hasattr(L, sym)
