"""Location of the reference source tree, for the build recipes and tests
that read it (oracle/build_ref.py, baseline/install_ref.py, the live
comparisons in tests/).  Nothing on the product path reads it.

The tree is taken from the PACKING_REFERENCE environment variable; the
default below is the one place that names where this container mounts it.
Where the tree is absent (a GPU box), the callers skip their reference
steps and use what was built or recorded from it beforehand.
"""
from __future__ import annotations

import os

ENV = "PACKING_REFERENCE"
DEFAULT = "/root/reference"


def reference_dir() -> str:
    return os.environ.get(ENV, DEFAULT)


def reference_core() -> str:
    return os.path.join(reference_dir(), "core")


def available() -> bool:
    return os.path.isdir(reference_core())
