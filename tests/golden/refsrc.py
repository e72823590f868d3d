"""Where the lightsmith sources are read from when a fixture is made or a plugin test runs here.

``LIGHTSMITH_SRC`` overrides the default checkout below; ``shim/`` supplies ``array_api_compat``, which the
sources import and which is not installed here. The GPU host has no lightsmith: the tests that need it skip.
"""

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = os.environ.get("LIGHTSMITH_SRC", "/root/reference/src")


def add_to_path(src: str = REF_SRC) -> bool:
    """Put the lightsmith sources (and the shim) on sys.path; False when they are not there."""
    if not os.path.isdir(os.path.join(src, "lightsmith")):
        return False
    for p in (src, os.path.join(HERE, "shim")):
        if p not in sys.path:
            sys.path.insert(0, p)
    return True
