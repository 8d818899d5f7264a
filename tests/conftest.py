import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


_SYSTEMS = {}


def get_system(name, **over):
    """Seeded synthetic system by name (cached per process)."""
    from pci_b200 import system as S
    key = (name, tuple(sorted(over.items())))
    if key not in _SYSTEMS:
        kw = S.CONFIGS[name]()
        kw.update(over)
        _SYSTEMS[key] = S.make_system(**kw)
    return _SYSTEMS[key]


_ORACLE_H = {}


def oracle_h(name, **over):
    """Oracle (rowptr, col, val, numzero, hmin, pairs) and J^2 CSR for a system (cached)."""
    import oracle as O
    key = (name, tuple(sorted(over.items())))
    if key not in _ORACLE_H:
        s = get_system(name, **over)
        o = O.Oracle(s)
        _ORACLE_H[key] = (o.form_h(), o.form_j())
    return _ORACLE_H[key]
