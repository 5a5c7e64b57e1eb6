"""Where the checkers find the reference solver's sources.  TEST INFRASTRUCTURE.

One setting: the environment variable DSMC_REFERENCE_SOURCES, else the
read-only reference checkout of the build machine.  The oracle/_ref recipe
(oracle/Makefile), build() and the tests that read the reference's own
files resolve it here; on a machine without the checkout they skip what
needs it, and nothing in the engine reads it.
"""
from __future__ import annotations

import os
from pathlib import Path

REFERENCE_SOURCES = Path(os.environ.get("DSMC_REFERENCE_SOURCES", "/root/reference"))


def reference_available() -> bool:
    """True when the reference's sources are present (its Boundary.cpp)."""
    return (REFERENCE_SOURCES / "src" / "Boundary.cpp").exists()
