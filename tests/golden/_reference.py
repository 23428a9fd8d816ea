"""Where the fixture scripts find the reference checkout: the first
command-line argument, else the ``FBALP_REFERENCE`` environment variable."""

from __future__ import annotations

import os
from pathlib import Path


def reference_root() -> Path:
    root = os.environ.get("FBALP_REFERENCE")
    if not root:
        raise SystemExit("pass the reference checkout as the first argument or set FBALP_REFERENCE")
    return Path(root)
