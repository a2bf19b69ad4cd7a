"""The device-memory and batch entry points the Julia shim binds (CDFTB200.jl), through
the C ABI: cdft_converge_dev on a caller's stream (cdft_plan_set_stream) equals
cdft_converge, cdft_batch_converge_dev equals cdft_batch_converge, and the snapshot hook
(DFTProblem's save_callback, converge.jl:31-60,256-267) hands out the iterate every k
evaluations without changing the result."""
import ctypes

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu

KW = dict(beta=0.1, tol=1e-10, anderson_m=5)


def test_converge_dev_on_caller_stream_equals_host_path():
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib
    lib = _lib.load()
    sp, _ = S.slit_pore(4e-9, 1e5, 180)
    r0 = cd.initialize_profiles(sp)
    host = r0.copy()
    res_h = cd.converge(sp, host, engine="grid", **KW)
    stream = torch.cuda.Stream()
    _lib.check(lib.cdft_plan_set_stream(sp._plan, ctypes.c_void_p(stream.cuda_stream)))
    dev = torch.from_numpy(r0.copy()).cuda()
    opts = cd.AASol.for_system(sp, **KW).c_opts(engine="grid")
    res = _lib.Result()
    _lib.check(lib.cdft_converge_dev(sp._plan, ctypes.c_void_p(dev.data_ptr()), ctypes.byref(opts), ctypes.byref(res)))
    stream.synchronize()
    _lib.check(lib.cdft_plan_set_stream(sp._plan, None))
    assert res.errcode == res_h.errcode == 0 and res.evaluations == res_h.evaluations
    assert np.array_equal(dev.cpu().numpy(), host)


def test_batch_converge_dev_equals_host_batch():
    import torch
    import cdft_b200 as cd
    from cdft_b200 import _lib
    lib = _lib.load()
    systems = [S.slit_pore(H, p, N)[0] for H, p, N in [(2e-9, 1e3, 100), (5e-9, 1e6, 250), (8e-9, 1e7, 400)]]
    r0 = [cd.initialize_profiles(s) for s in systems]
    host = [r.copy() for r in r0]
    res_h = cd.batch_converge(systems, host, **KW)
    dev = [torch.from_numpy(r.copy()).cuda() for r in r0]
    n = len(systems)
    plans = (ctypes.c_void_p * n)(*[s._plan.value for s in systems])
    ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in dev])
    opts = cd.AASol.for_system(systems[0], **KW).c_opts()
    res = (_lib.Result * n)()
    torch.cuda.synchronize()
    _lib.check(lib.cdft_batch_converge_dev(plans, n, ptrs, ctypes.byref(opts), res))
    for k in range(n):
        assert res[k].errcode == res_h[k].errcode == 0 and res[k].evaluations == res_h[k].evaluations
        assert np.array_equal(dev[k].cpu().numpy(), host[k])


def test_snapshot_hook_every_k_evaluations():
    import cdft_b200 as cd
    sp, _ = S.slit_pore(4e-9, 1e5, 180)
    r0 = cd.initialize_profiles(sp)
    plain = r0.copy()
    res_p = cd.converge(sp, plain, engine="grid", **KW)
    seen = []
    hooked = r0.copy()
    res = cd.converge(sp, hooked, save_interval=5, save_callback=lambda it, rho: seen.append((it, rho)), **KW)
    assert res.evaluations == res_p.evaluations and np.array_equal(hooked, plain)
    its = [it for it, _ in seen]
    assert its == list(range(5, 5 * len(its) + 1, 5)) and len(its) >= res.evaluations // 5 - 1
    for it, rho in seen:
        assert rho.shape == r0.shape and np.all(rho > 0)
    assert not np.array_equal(seen[0][1], seen[-1][1])   # the iterate moves between snapshots
