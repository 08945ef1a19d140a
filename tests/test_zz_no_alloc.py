"""psod_cic_rho_static: the CIC density entry point that allocates nothing.

Some host codes cannot let this library allocate device memory: drivers that
size all of the GPU's memory themselves (several MPI ranks sharing one GPU
under fixed per-rank budgets, or a host whose own pool allocator owns the
device) and forbid libraries from calling cudaMalloc.  For them
psod_cic_rho_static computes the per-particle density of psod_cic +
psod_cicm1 with its node grid in a static device array (zones up to 64 cells
per side).  Both paths sum the CIC weights in int64 fixed point at 2^-40 in
the reference's term order, so the result must equal the oracle's canonical
density bit for bit, on every call (the shared array keeps the previous
call's nodes and must be cleared each time).

This file runs last so that a failure here leaves every other test already
run; it passes alone in a fresh process and after the other tests.
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

RTOL = 1e-6  # the density tolerance of the parity tests (reference arithmetic)


def static_rho(lib, pos, nx, nxbuffer, bad):
    n = pos.shape[0]
    rho = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.psod_cic_rho_static(n, C.c_void_p(pos.data_ptr()), nx, 0, nxbuffer, C.c_void_p(rho.data_ptr()),
                                 C.c_void_p(bad.data_ptr()), C.c_void_p(stream))
    assert st == capi.OK
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
    return rho.cpu().numpy()


# nx = 32 with the default buffer (nx/2); nx = 24 (not a power of two, so the
# CIC cell spacing 1/(2nx) is inexact) with a buffer of 5 cells
@pytest.mark.parametrize("nx,nxbuffer,seed", [(32, 0, 41), (24, 5, 42)])
def test_static_rho_equals_oracle_and_context_path_twice(oracle, nx, nxbuffer, seed):
    b = synth.make_box(nx, nmax_halo=2000, seed=seed)
    pos_h = b.pos.numpy()
    p = oracle.Params(nx=nx, nxbuffer=nxbuffer)
    rho_can = oracle.rho(p, pos_h, oracle.CANONICAL)
    rho_ref = oracle.rho(p, pos_h, oracle.REFERENCE)
    s = SphericalOverdensity(nx, nxbuffer=nxbuffer)
    s.load(pos_h, b.ids.numpy())
    s.cic()
    rho_ctx = s.cicm1()
    s.close()
    assert np.array_equal(rho_ctx, rho_can)

    lib = capi.load()
    pos = b.pos.cuda().contiguous()
    bad = torch.ones(1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # two calls in a row: the second starts from the first's nodes
        rho = static_rho(lib, pos, nx, nxbuffer, bad)
        assert np.array_equal(rho, rho_can)
        assert np.array_equal(rho, rho_ctx)
        np.testing.assert_allclose(rho, rho_ref, rtol=RTOL, atol=0)


def test_static_rho_rejects_oversized_zone_and_host_pointers():
    lib = capi.load()
    pos = torch.rand(1000, 3, device="cuda")
    rho = torch.zeros(1000, dtype=torch.float64, device="cuda")
    args = (C.c_void_p(pos.data_ptr()), 65, 0, 0, C.c_void_p(rho.data_ptr()), None, None)
    assert lib.psod_cic_rho_static(1000, *args) == capi.ERR_ARG
    host = np.zeros(3000, np.float32)
    assert lib.psod_cic_rho_static(1000, C.c_void_p(host.ctypes.data), 16, 0, 0, C.c_void_p(rho.data_ptr()), None,
                                   None) == capi.ERR_ARG
