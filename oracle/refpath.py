"""Location of the GraphWalker reference tree, for the recipes that build the
checker (oracle/Makefile `ref`, the drop-in apps of graphwalker_b200/compat)
and the golden fixtures: the GW_REFERENCE environment variable, else the
default below.  This is the one place that default is written; the
Makefiles take the tree from REF= or GW_REFERENCE.  The tree is read only
where it exists (it is absent where the prebuilt files are used)."""
from __future__ import annotations

import os
from pathlib import Path

DEFAULT = "/root/reference"
REFERENCE = Path(os.environ.get("GW_REFERENCE") or DEFAULT)
