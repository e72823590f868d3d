"""Where the lightsmith sources are imported from when a fixture is made or a test runs lightsmith's own code.

The default is the reference install under ``baseline/_ref`` (``python baseline/install_ref.py``), which holds
the unmodified ``lightsmith`` package and the ``array_api_compat`` stand-in and travels with the working tree;
``LIGHTSMITH_SRC`` names another directory that holds a ``lightsmith`` package. Tests that need lightsmith skip
where neither is present.
"""

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_SRC = os.environ.get("LIGHTSMITH_SRC", os.path.join(REPO, "baseline", "_ref"))


def add_to_path(src: str = REF_SRC) -> bool:
    """Put the lightsmith sources (and the ``array_api_compat`` stand-in) on sys.path; False when they are not
    there."""
    if not os.path.isdir(os.path.join(src, "lightsmith")):
        return False
    for p in (src, os.path.join(HERE, "shim")):
        if p not in sys.path:
            sys.path.insert(0, p)
    return True
