"""B200-native langevinfts chain-propagator solver.

`langevinfts_b200.langevinfts` is the drop-in pybind11 module (same classes and
methods as the reference's `langevinfts`); put this directory on sys.path, or
`from langevinfts_b200 import langevinfts`, to use it from the existing SCFT and
L-FTS drivers.  `langevinfts_b200.capi` binds the C ABI (include/lfts_b200.h).
"""
import os as _os

LIB_DIR = _os.path.dirname(_os.path.abspath(__file__))
