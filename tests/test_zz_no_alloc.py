"""psod_cic_rho_static: the CIC density entry point that allocates nothing.

Some callers cannot let this library allocate device memory: code recording
a stream into a CUDA graph (cudaMalloc is not allowed during capture) and host
codes that size all device memory themselves.  For them psod_cic_rho_static
computes the per-particle density of psod_cic + psod_cicm1 in a node grid
held in a static device array (zones up to 64 cells per side).  This file
runs last so that a failure here leaves every other test already run; it
passes alone in a fresh process and after the other tests.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from psod_b200 import capi, synth  # noqa: E402
from psod_b200.sod import SphericalOverdensity  # noqa: E402

RTOL = 1e-6  # the density tolerance of the parity tests


def test_static_rho_matches_context_path_twice():
    nx = 32
    b = synth.make_box(nx, nmax_halo=2000, seed=41)
    s = SphericalOverdensity(nx)
    s.load(b.pos.numpy(), b.ids.numpy())
    s.cic()
    rho_ref = s.cicm1()
    s.close()

    lib = capi.load()
    pos = b.pos.cuda().contiguous()
    n = pos.shape[0]
    bad = torch.ones(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the shared array keeps the previous call's nodes
        rho = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
        st = lib.psod_cic_rho_static(n, C.c_void_p(pos.data_ptr()), nx, 0, 0, C.c_void_p(rho.data_ptr()),
                                     C.c_void_p(bad.data_ptr()), C.c_void_p(stream))
        assert st == capi.OK
        torch.cuda.synchronize()
        assert int(bad.item()) == 0
        np.testing.assert_allclose(rho.cpu().numpy(), rho_ref, rtol=RTOL, atol=0)


def test_static_rho_rejects_oversized_zone_and_host_pointers():
    lib = capi.load()
    pos = torch.rand(1000, 3, device="cuda")
    rho = torch.zeros(1000, dtype=torch.float64, device="cuda")
    args = (C.c_void_p(pos.data_ptr()), 65, 0, 0, C.c_void_p(rho.data_ptr()), None, None)
    assert lib.psod_cic_rho_static(1000, *args) == capi.ERR_ARG
    host = np.zeros(3000, np.float32)
    assert lib.psod_cic_rho_static(1000, C.c_void_p(host.ctypes.data), 16, 0, 0, C.c_void_p(rho.data_ptr()), None,
                                   None) == capi.ERR_ARG
