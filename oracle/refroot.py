"""Where the reference project's sources are, for the checker builds only.

The checker libraries under oracle/_ref are compiled from the reference's own
sources where they lie.  Their location comes from the environment variable
PPPM_REFERENCE_ROOT, else from the "reference_path" entry of the repository's
BASELINE.json; with neither (or a path that does not exist, as on a host that
only runs the prebuilt checkers) there is nothing to build.
"""
from __future__ import annotations

import json
import os

_REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root():
    """Directory of the reference's sources, or None when they are absent."""
    cand = os.environ.get("PPPM_REFERENCE_ROOT")
    if not cand:
        try:
            with open(os.path.join(_REPO, "BASELINE.json")) as f:
                cand = json.load(f).get("reference_path")
        except (OSError, ValueError):
            cand = None
    return cand if cand and os.path.isdir(cand) else None
