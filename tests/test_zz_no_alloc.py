"""The allocation-free energy entry point, fabipb_b200_energy_noalloc, against
fabipb_b200_energy through the C ABI (include/fabipb_b200.h).

It is kept in its own file, collected after the other GPU tests, and passes
both there and alone in a fresh process: the fixed scratch array it uses is
looked up on the first call in the process, and every later call reuses it
with the previous call's partial sums still in it.

Tolerance: relative 1e-12 (the FP64 energy tolerance of the parity tests);
both entry points run the same walk and the same sequential sum.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import case_params
from fabipb_b200 import lib, meshio
import make_golden

pytestmark = pytest.mark.gpu


def _entry():
    f = lib.load().fabipb_b200_energy_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("name", ["sphere1280", "star2048"])
def test_energy_noalloc_matches_energy(name, case_dir, golden_meta):
    import torch

    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    s = lib.Surface(pan, lib.params(precision=lib.FP64, **case_params(golden_meta[name]["opts"])))
    s.set_charges(ch)
    f = _entry()
    sig1 = make_golden.seeded_sigma(s.n, seed=0)
    sig2 = make_golden.seeded_sigma(s.n, seed=1)
    d_sig = torch.from_numpy(sig1).to("cuda")
    d_raw = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    # no charge tree yet: refused with a message, nothing launched
    assert f(s.h, d_sig.data_ptr(), d_raw.data_ptr()) == 0
    assert "charge tree" in lib.last_error()

    ref1 = s.energy_raw(sig1)           # the existing entry point (builds the tree)
    ref2 = s.energy_raw(sig2)
    assert ref1 != ref2

    # two calls in a row on different densities: the second must not see the first's partial sums
    for sig, ref in ((sig1, ref1), (sig2, ref2)):
        d_sig.copy_(torch.from_numpy(sig))
        d_raw.fill_(float("nan"))
        torch.cuda.synchronize()
        assert f(s.h, d_sig.data_ptr(), d_raw.data_ptr()) == 1, lib.last_error()
        torch.cuda.synchronize()
        got = float(d_raw.cpu()[0])
        assert abs(got - ref) <= 1e-12 * abs(ref), (got, ref)
    s.close()
