"""Module alias so code written against the reference extension imports this
one unchanged: after ``install_alias()``, ``from cudaForwardBackwardRenderer
import _C`` (reference ``Renderer.py:5``) yields ``word2world_b200._C``."""
from __future__ import annotations

import sys
import types

from . import _C


def install_alias(name: str = "cudaForwardBackwardRenderer") -> types.ModuleType:
    pkg = types.ModuleType(name)
    pkg._C = _C
    pkg.__path__ = []  # a package, so "name._C" resolves
    sys.modules[name] = pkg
    sys.modules[name + "._C"] = _C
    return pkg
