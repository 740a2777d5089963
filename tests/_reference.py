"""Import of the ceres-torch package itself for the drop-in tests.

The package is looked up in ``baseline/_ref`` (an offline ``pip install --target``
of ceres-torch into this repository, git-ignored) or in the directory named by
``CERES_TORCH_REFERENCE``; tests that need it are skipped when neither exists.
"""
from __future__ import annotations

import importlib
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def reference_module():
    """The ``ceres_torch`` module, or None when it is not installed."""
    candidates = [os.environ.get("CERES_TORCH_REFERENCE"), str(ROOT / "baseline" / "_ref")]
    for c in candidates:
        if c and (Path(c) / "ceres_torch" / "__init__.py").exists():
            if c not in sys.path:
                sys.path.append(c)
            try:
                return importlib.import_module("ceres_torch")
            except ImportError:
                return None
    return None
