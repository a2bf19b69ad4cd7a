"""GPU test of the allocation-free functional derivative.

Callers whose device memory is owned by a pool or caching allocator (or that
forbid device allocations after start-up) cannot let a library call
cudaMalloc; cdft_functional_derivative_noalloc serves them from a fixed
scratch array inside the library.  Its result must equal the plan-based
cdft_functional_derivative_dev on the same inputs, call after call, without
changing the device's free memory.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def _noalloc(sysp, rho_dev, out_dev):
    from cdft_b200 import _lib
    lib = _lib.load()
    return lib.cdft_functional_derivative_noalloc(ctypes.byref(sysp._desc), ctypes.c_void_p(rho_dev.data_ptr()),
                                                  ctypes.c_void_p(out_dev.data_ptr()), None)


def _reference_path(sysp, rho_dev):
    import torch
    from cdft_b200 import _lib
    lib = _lib.load()
    out = torch.empty_like(rho_dev)
    _lib.check(lib.cdft_functional_derivative_dev(sysp._plan, ctypes.c_void_p(rho_dev.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr())))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_plan_path_twice():
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib
    rng = np.random.default_rng(7)
    # different systems: a call must not depend on what the one before left in the scratch.
    # The third (4096 points, two components) is the largest the scratch takes: its
    # convolutions are split over 4 tap chunks whose partial sums meet in the scratch.
    cases = [S.water_octane_lle(N=256)[0], S.methane_wall(N=201)[0], S.water_octane_lle(N=4096)[0]]
    rhos = [S.random_smooth_profile(cases[0], rng), cd.initialize_profiles(cases[1]),
            S.random_smooth_profile(cases[2], rng)]
    rho_dev = [torch.from_numpy(np.ascontiguousarray(r)).cuda() for r in rhos]
    expect = [_reference_path(sp, r) for sp, r in zip(cases, rho_dev)]
    out_dev = [torch.full_like(r, float("nan")) for r in rho_dev]
    torch.cuda.synchronize()
    # calls in a row
    _lib.check(_noalloc(cases[0], rho_dev[0], out_dev[0]))
    free_before = torch.cuda.mem_get_info()[0]
    _lib.check(_noalloc(cases[1], rho_dev[1], out_dev[1]))
    _lib.check(_noalloc(cases[2], rho_dev[2], out_dev[2]))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before   # the later calls allocated nothing
    for sp, e, o in zip(cases, expect, out_dev):
        got = o.cpu().numpy()
        for i in range(sp.nc):
            scale = np.max(np.abs(e[i]))
            assert np.max(np.abs(got[i] - e[i])) <= 1e-10 * scale


def test_noalloc_rejects_oversized_system():
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib
    sysp, _ = S.slit_pore(8e-9, 1e5, N=_lib.NOALLOC_MAX_N + 1)
    rho_dev = torch.from_numpy(cd.initialize_profiles(sysp)).cuda()
    out_dev = torch.empty_like(rho_dev)
    rc = _noalloc(sysp, rho_dev, out_dev)
    assert rc == _lib.E_UNSUPPORTED
    buf = ctypes.create_string_buffer(256)
    _lib.load().cdft_last_error(buf, 256)
    assert b"too large" in buf.value
