"""pytest plugin that runs pyising's own test suite against this backend.

    PYISING_REFERENCE_SRC=<pyising>/src PYTHONPATH=<this repo>/tests \\
        python -m pytest -p reference_plugin <pyising>/tests/test_backends.py -k "b200 or set_beta"

It registers the B200 backend into the pyising source tree named by PYISING_REFERENCE_SRC
(``register_with_pyising``) before pyising's tests build their parametrisation from
``REGISTRY`` (tests/test_backends.py:11-12), and puts the ``b200`` keys first, so the cases that
take only the first int8 and msc backend (``INT8[:1] + MSC[:1]``, the set_beta test) run on it.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

_SRC = os.environ.get("PYISING_REFERENCE_SRC")
if not _SRC or not Path(_SRC).is_dir():
    raise RuntimeError("PYISING_REFERENCE_SRC must name pyising's src folder")
sys.path.insert(0, _SRC)
sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

import pyising_b200  # noqa: E402

_pb = pyising_b200.register_with_pyising()
_items = list(_pb.REGISTRY.items())
_pb.REGISTRY.clear()
_pb.REGISTRY.update({k: v for k, v in _items if k[0] == "b200"})
_pb.REGISTRY.update({k: v for k, v in _items if k[0] != "b200"})
_pb.load.cache_clear()
