"""ps_density_solve_device_noalloc: the contour density for callers that
cannot allocate device memory (for example code that runs inside a host
program whose own pool owns all device memory, or a loop that cannot take the
synchronisation of cudaMalloc / cudaFree).  It keeps its contour-weight table
in a fixed device array of the library instead of allocating one per call.

Checked here through the C ABI against ps_density_solve_device, which
allocates its table: two calls in a row with different rules and lengths (the
second must overwrite the first call's table), on torch's current stream.
This file is collected last on purpose; it passes alone in a fresh process
(the first call on the device sets up the table address) and after the rest.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    from polystring_b200 import capi
    return torch, capi, capi.load()


def _call(lib, fn, rule, q, qc, ds, cc, phi, stream):
    return getattr(lib, fn)(rule, q.data_ptr(), qc.data_ptr(), q.shape[0], phi.numel(), ds, cc, phi.data_ptr(),
                            stream)


# (rule, len): every contour rule at the shortest length its precondition
# allows and at a longer one; consecutive calls change rule and length, so
# each call must overwrite the previous call's table
CASES = [("trapezoid", 2), ("trapezoid", 40), ("simpson", 5), ("simpson", 51), ("quad4_closed", 8),
         ("quad4_closed", 38), ("quad4_open", 10), ("quad4_open", 47), ("quad4_semiopen_left", 9),
         ("quad4_semiopen_left", 33), ("quad4_semiopen_right", 9), ("quad4_semiopen_right", 60)]


def test_noalloc_density_matches_allocating_entry_point_twice(env):
    """Every rule, each run twice in a row (the first call of a pair follows a
    call of another rule or length), against the allocating entry point."""
    torch, capi, lib = env
    dev = torch.device("cuda:0")
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    gen = torch.Generator(device="cpu").manual_seed(11)
    shapes = [(32, 16, 8), (24, 12, 10)]
    for i, (name, length) in enumerate(CASES):
        rule = capi.RULES[name]
        shape = shapes[i % 2]
        ds, cc = 0.5 / length, 0.7 + 0.1 * i
        q = (1 + 0.1 * torch.randn((length,) + shape, generator=gen, dtype=torch.float64)).to(dev)
        qc = (1 + 0.1 * torch.randn((length,) + shape, generator=gen, dtype=torch.float64)).to(dev)
        ref = torch.zeros(shape, dtype=torch.float64, device=dev)
        capi.check(_call(lib, "ps_density_solve_device", rule, q, qc, ds, cc, ref, stream))
        for rep in range(2):
            out = torch.full(shape, float("nan"), dtype=torch.float64, device=dev)
            capi.check(_call(lib, "ps_density_solve_device_noalloc", rule, q, qc, ds, cc, out, stream))
            torch.cuda.synchronize(dev)
            r, o = ref.cpu().numpy(), out.cpu().numpy()
            assert np.isfinite(o).all()
            assert np.abs(o - r).max() < 1e-13, (name, length, rep)


def test_noalloc_density_rejects_what_it_cannot_hold(env):
    torch, capi, lib = env
    dev = torch.device("cuda:0")
    big = capi.PS_DENSITY_NOALLOC_MAX_LEN + 1
    q = torch.ones((big, 4), dtype=torch.float64, device=dev)
    phi = torch.zeros(4, dtype=torch.float64, device=dev)
    rc = _call(lib, "ps_density_solve_device_noalloc", capi.RULES["trapezoid"], q, q, 0.01, 1.0, phi, None)
    assert rc == capi.PS_ERR_INVALID
    assert str(capi.PS_DENSITY_NOALLOC_MAX_LEN) in lib.ps_last_error().decode()
    # a rule whose precondition fails is the same error as the allocating entry point's
    q = torch.ones((36, 4), dtype=torch.float64, device=dev)
    rc = _call(lib, "ps_density_solve_device_noalloc", capi.RULES["simpson"], q, q, 0.01, 1.0, phi, None)
    assert rc == _call(lib, "ps_density_solve_device", capi.RULES["simpson"], q, q, 0.01, 1.0, phi, None)
    assert rc == capi.PS_ERR_QUADRATURE
