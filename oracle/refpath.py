"""TEST INFRASTRUCTURE ONLY: where the reference checkout lies.

The reference's sources and data files (hadalhw17/RayEngine) are read only to
build oracle/_ref/ (the reference's own host code) and by tests that compare
against its shipped meshes.  The location comes from the environment variable
RAYENGINE_REFERENCE; without it, the default checkout location below is used
when it exists.  Everything that needs the reference skips when neither is
present (the GPU machines carry only the prebuilt oracle/_ref/ libraries).
"""
from __future__ import annotations

import os

ENV = "RAYENGINE_REFERENCE"
_DEFAULT = "/root/reference"


def reference_root():
    """The reference checkout (a directory holding RayEngine/ and Sandbox/), or None."""
    p = os.environ.get(ENV) or _DEFAULT
    return p if os.path.isdir(os.path.join(p, "RayEngine")) else None


def reference_file(*parts):
    """A path inside the reference checkout, or None when it is absent."""
    root = reference_root()
    if root is None:
        return None
    p = os.path.join(root, *parts)
    return p if os.path.exists(p) else None
