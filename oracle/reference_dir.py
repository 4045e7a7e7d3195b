"""Location of the reference source tree, for the recipes that compile or
read it (the oracle's reference harness, the golden-vector script, the
compile-unchanged test of the reference's example).  TEST INFRASTRUCTURE.

One environment variable, KITES_REFERENCE_DIR, names it; when it is unset
the build container's read-only mount is assumed.  Callers treat a missing
tree as "not available" and skip: nothing that runs on a GPU box reads it.
"""
from __future__ import annotations

import os

REFERENCE_DIR = os.environ.get("KITES_REFERENCE_DIR", "/root/reference")


def reference_dir() -> str | None:
    """The reference tree if it is present (it holds kites/), else None."""
    return REFERENCE_DIR if os.path.isdir(os.path.join(REFERENCE_DIR, "kites")) else None
