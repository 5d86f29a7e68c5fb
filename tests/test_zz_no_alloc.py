"""The allocation-free laplc entry point (mpg_laplc_noalloc) against the ordinary one.

mpg_laplc_noalloc serves callers that may not allocate device memory when they call in: host
programs whose memory pool owns the whole GPU (so a stray cudaMalloc could fail or unbalance the
pool) and time-critical loops where cudaMalloc/cudaFree would stall the device.  Its scratch is
a static device array; this test drives it through the C ABI twice in a row and checks each
result against mpg_laplc on the same input.  It lives in its own file, collected last, and
passes both alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from src_b200 import api, mesh
from src_b200.cabi import F_WORK, RunParams

pytestmark = pytest.mark.gpu


def _laplc_noalloc(s, dev_in, dev_out, impfl):
    rc = api.lib().mpg_laplc_noalloc(s.h, C.c_void_p(dev_in.data_ptr()), C.c_void_p(dev_out.data_ptr()), impfl)
    if rc != 0:
        raise api.MpgError(rc, api.lib().mpg_last_error().decode())
    s.synchronize()


def test_laplc_noalloc_matches_laplc():
    import torch
    cm = mesh.generate(48, L=41, seed=0)          # 94,464 nodes, within the static scratch
    rm = cm.to_reference()
    rng = np.random.default_rng(11)
    with api.Solver(RunParams(delt=10.0), rm) as s:
        for call, impfl in enumerate((1, 0)):       # two calls in a row
            p = rng.standard_normal(rm.npoin)
            s.set(F_WORK, p)
            s.laplc(F_WORK, F_WORK + 1, impfl)
            expected = s.get(F_WORK + 1)
            dev_in = torch.tensor(p, dtype=torch.float64, device="cuda")
            dev_out = torch.full((rm.npoin,), np.nan, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            _laplc_noalloc(s, dev_in, dev_out, impfl)
            got = dev_out.cpu().numpy()
            # same kernels and same summation order: equal to the last bit (the other tests'
            # operator tolerance is exact equality too)
            assert np.array_equal(got, expected), f"call {call}"


def test_laplc_noalloc_rejects_large_mesh():
    import torch
    cm = mesh.generate(60, L=41, seed=0)          # 147,600 nodes > MPG_NOALLOC_MAX_NODES
    rm = cm.to_reference()
    with api.Solver(RunParams(delt=10.0), rm) as s:
        a = torch.zeros(rm.npoin, dtype=torch.float64, device="cuda")
        b = torch.zeros(rm.npoin, dtype=torch.float64, device="cuda")
        with pytest.raises(api.MpgError) as e:
            _laplc_noalloc(s, a, b, 1)
        assert e.value.code == 1 and "static scratch" in str(e.value)
