"""The reference's module name: ``import cccollisions`` as a caller of the reference
extension writes it (module ``cccollisions``, ``setup.py:17,21``; functions
``src/cccollisions.cpp:426-468``).

Every name is the B200 implementation from ``cccollisions_b200``: the same functions,
argument names, defaults, output shapes and dtypes as the reference's pybind module.
"""
from cccollisions_b200 import *  # noqa: F401,F403
from cccollisions_b200 import __all__  # noqa: F401
