"""Where the reference source tree is -- TEST INFRASTRUCTURE ONLY.

The reference's own solver sources are compiled into oracle/_ref (by
``make -C oracle ref REFROOT=<tree>``) and read by the fixture generator in
tests/golden.  Neither the library nor the tests read the tree at run time.

The tree is taken from the environment variable IMEXLB_REFERENCE, else from
the ``reference_path`` key of BASELINE.json at the repository root; None
when neither names an existing directory.
"""
from __future__ import annotations

import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root() -> str | None:
    cand = os.environ.get("IMEXLB_REFERENCE")
    if not cand:
        try:
            with open(os.path.join(ROOT, "BASELINE.json")) as fh:
                cand = json.load(fh).get("reference_path")
        except (OSError, ValueError):
            cand = None
    return cand if cand and os.path.isdir(cand) else None
