"""Loader for the reference's own `langevinfts` module built by oracle/Makefile
(oracle/_ref, CPU platform "cpu-mkl" with the project FFT shim).  Test
infrastructure only: it is loaded under a private name so that it can sit next
to the product module in one process."""
import glob
import importlib.machinery
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_mod = None


def path():
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "langevinfts*.so"))
    return hits[0] if hits else None


def load():
    """The reference module, or None when oracle/_ref has not been built."""
    global _mod
    if _mod is None:
        p = path()
        if p is None:
            return None
        loader = importlib.machinery.ExtensionFileLoader("langevinfts", p)
        spec = importlib.util.spec_from_file_location("langevinfts", p, loader=loader)
        m = importlib.util.module_from_spec(spec)
        loader.exec_module(m)
        _mod = m
    return _mod
