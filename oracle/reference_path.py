"""TEST INFRASTRUCTURE -- where the read-only reference checkout lies.

The checkout is needed only to BUILD the checker (oracle/ref compiles the
reference's own sources) and to read the particle files it ships; nothing
that runs on a GPU machine reads it. The location is $FS_REFERENCE_DIR, and
DEFAULT below when that variable is unset. This file is the one place that
names the default; the Makefiles take it as REF=... from their caller.
"""
from __future__ import annotations

import os

DEFAULT = "/root/reference"


def reference_dir() -> str:
    return os.environ.get("FS_REFERENCE_DIR", DEFAULT)


def present() -> bool:
    """Whether the checkout (its libFluid sources) is there to build from."""
    return os.path.isdir(os.path.join(reference_dir(), "src", "libFluid"))
