"""The allocation-free energy entry point, fabipb_b200_energy_noalloc, against
fabipb_b200_energy through the C ABI (include/fabipb_b200.h).

It is kept in its own file, collected after the other GPU tests, and passes
both there and alone in a fresh process: the fixed scratch array it uses is
looked up in the current CUDA context on every call, and every call reuses it
with the previous call's partial sums still in it.

Checked, in FP64 and in mixed contexts (whose energy walk is the FP32-term
instantiation of the same kernel): two calls in a row on different densities
equal the existing entry point's energies; device memory in use is the same
before and after the calls (nothing allocated); a call queued on a
non-default stream set with fabipb_b200_set_stream gives the same result.

Tolerance: relative 1e-12 (the FP64 energy tolerance of the parity tests);
both entry points run the same walk and the same fixed-order sum.
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


@pytest.mark.parametrize("precision", [lib.FP64, lib.MIXED])
@pytest.mark.parametrize("name", ["sphere1280", "star2048"])
def test_energy_noalloc_matches_energy(name, precision, case_dir, golden_meta):
    import torch

    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    s = lib.Surface(pan, lib.params(precision=precision, **case_params(golden_meta[name]["opts"])))
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

    # two calls in a row on different densities: the second must not see the
    # first's partial sums; device memory in use does not change
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for sig, ref in ((sig1, ref1), (sig2, ref2)):
        d_sig.copy_(torch.from_numpy(sig))
        d_raw.fill_(float("nan"))
        torch.cuda.synchronize()
        assert f(s.h, d_sig.data_ptr(), d_raw.data_ptr()) == 1, lib.last_error()
        torch.cuda.synchronize()
        got = float(d_raw.cpu()[0])
        assert abs(got - ref) <= 1e-12 * abs(ref), (got, ref)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, "device memory in use changed by %d bytes" % (free0 - free1)

    # on a caller's non-default stream: inputs written on that stream, the
    # call queued behind them, the result read after that stream
    side = torch.cuda.Stream()
    s.set_stream(side.cuda_stream)
    with torch.cuda.stream(side):
        d_sig.copy_(torch.from_numpy(sig1).to("cuda", non_blocking=False))
        d_raw.fill_(float("nan"))
    assert f(s.h, d_sig.data_ptr(), d_raw.data_ptr()) == 1, lib.last_error()
    side.synchronize()
    got = float(d_raw.cpu()[0])
    assert abs(got - ref1) <= 1e-12 * abs(ref1), (got, ref1)
    s.close()
