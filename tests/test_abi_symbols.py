"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "cuda-fabipb_b200", "lib", "libfabipb_b200.so")
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in DECL.finditer(text):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_header_declares_plugin_abi():
    names = declared_functions()
    for sym in ("gpuBackendAvailable", "gpuNearfieldLastError", "gpuM2LLastError", "gpuNearfieldApply",
                "gpuDirectApply", "gpuM2LApply", "gpuQ2MApply", "gpuL2PApply", "gpuReleaseMatvecCaches",
                "gpuReleaseChargeTreeCache", "gpuSetupRHS", "gpuPanelChargeTreeEnergy", "gpuRhsReuseCoulombDot",
                "gpuRhsReusePanelChargeTreeEnergy", "gpuChargeTreeRHS", "gpuBuildPrecondPairsBatched",
                "gpuBuildPrecondDisjointBlock"):
        assert sym in names


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_library_reports_errors_without_a_context():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "cuda-fabipb_b200"))
    from fabipb_b200 import lib
    L = lib.load()
    assert L.fabipb_b200_matvec(None, 1.0, None, 0.0, None, 0) == 0
    assert len(lib.last_error()) > 0
