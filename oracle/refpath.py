"""Location of the reference checkout for the checkers that read it in place.

``NODALS_REFERENCE`` when set, else the default of ``REFROOT`` in
``oracle/Makefile`` (the one recipe that names it).  ``reference_root()``
returns None when that directory is absent (the GPU box has no reference
tree), and the steps that need it skip.
"""
from __future__ import annotations

import os
import re
from pathlib import Path
from typing import Optional

_MAKEFILE = Path(__file__).resolve().parent / "Makefile"


def _makefile_default() -> Optional[str]:
    m = re.search(r"^REFROOT\s*\?=\s*\$\(if [^,]*,[^,]*,([^)]*)\)", _MAKEFILE.read_text(), re.M)
    return m.group(1).strip() if m else None


def reference_root() -> Optional[Path]:
    env = os.environ.get("NODALS_REFERENCE")
    cand = env if env else _makefile_default()
    if not cand:
        return None
    p = Path(cand)
    return p if p.is_dir() else None
