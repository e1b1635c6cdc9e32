"""Location of the reference source tree, for the recipes and tests that read
it where it lies (read-only): the FALCOR_REF environment variable, else the
checkout this container mounts.  The GPU tests, smoke() and bench.py never
read the reference tree.

TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import os
from pathlib import Path

DEFAULT = "/root/reference"


def root() -> Path:
    """The reference checkout (the directory holding Source/, scripts/, tests/)."""
    return Path(os.environ.get("FALCOR_REF", DEFAULT))


def source() -> Path:
    return root() / "Source"


def present() -> bool:
    return source().is_dir()
