"""Drop-in support for the reference's own application sources.

The build steps and tests that read the reference's sources (to compile its
application mains against gswitch_b200/compat/gswitch.h, to convert its
selector trees, to build its CPU validators for oracle pinning) find the
reference tree through the GSW_REFERENCE_TREE environment variable.
"""
from __future__ import annotations

import os

_DEFAULT_TREE = "/root/reference"


def reference_tree() -> str:
    """Root of the reference source tree (may not exist, e.g. on a machine
    that only runs the prebuilt library)."""
    return os.environ.get("GSW_REFERENCE_TREE", _DEFAULT_TREE)
