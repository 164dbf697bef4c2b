"""dampm_cfl_dt_noalloc, the allocation-free CFL step, against the step's own
dt (dampm_status) on the same particle state.

Kept in its own file, named to be collected last, so that it runs both alone
and after every other GPU test.  Tolerance: exact (0 ulp) -- maxima do not
depend on the reduction order and the dt expression is the step's own.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.dampm_cfl_dt_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong,
                  C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_void_p, C.c_void_p]
    return f


def _host_dt(vpx, vpy, hp, g, CFL, hx, hy):
    """main/optim_par.cpp:289-304 evaluated in numpy (IEEE sqrt and divide)."""
    mvx, mvy, hmax = np.abs(vpx).max(), np.abs(vpy).max(), hp.max()
    a = np.sqrt(g * hmax) + mvx
    b = np.sqrt(g * hmax) + mvy
    cel = abs(b if a < b else a)
    return CFL * min(hx, hy) / (1e-2 + cel), cel, mvx, mvy, hmax


def test_cfl_dt_noalloc_matches_step_dt(cuda_lib):
    import torch
    from amsc_b200 import scenarios
    from amsc_b200.dampm import Solver

    assert torch.cuda.is_available()
    f = _bind(cuda_lib)
    d = scenarios.mudflow(N=256)
    sc = d.scalars
    g, CFL, hx, hy = sc["g"], sc["CFL"], sc["hx"], sc["hy"]
    stream = torch.cuda.current_stream().cuda_stream
    with Solver(d) as s:
        s.step(3)
        for _ in range(2):
            st = s.get_state()
            n = st["x"].shape[0]
            dev = {k: torch.from_numpy(st[k]).to("cuda") for k in ("vpx", "vpy", "hp")}
            outs = []
            for _call in range(2):  # two calls in a row on the same state
                out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
                rc = f(dev["vpx"].data_ptr(), dev["vpy"].data_ptr(), dev["hp"].data_ptr(),
                       n, g, CFL, hx, hy, out.data_ptr(), stream)
                assert rc == 0
                outs.append(out)
            torch.cuda.synchronize()
            got = [o.cpu().numpy() for o in outs]
            s.step(1)  # the existing entry point's dt for this state
            dt_step = s.status()["dt"]
            for v in got:
                assert v[0] == dt_step, (v[0], dt_step)
                assert tuple(v) == _host_dt(st["vpx"], st["vpy"], st["hp"], g, CFL, hx, hy)
            # a shorter call after a longer one reads none of the longer
            # call's partial maxima
            m = n // 3
            out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
            assert f(dev["vpx"].data_ptr(), dev["vpy"].data_ptr(), dev["hp"].data_ptr(),
                     m, g, CFL, hx, hy, out.data_ptr(), stream) == 0
            torch.cuda.synchronize()
            assert tuple(out.cpu().numpy()) == _host_dt(st["vpx"][:m], st["vpy"][:m],
                                                        st["hp"][:m], g, CFL, hx, hy)


def test_cfl_dt_noalloc_leaves_device_memory_alone(cuda_lib):
    """The point of the entry point: a call allocates and frees nothing, so the
    device's free memory is the same before and after a run of calls."""
    import torch
    f = _bind(cuda_lib)
    n = 3_000_000  # more blocks than the scratch holds partials for
    v = torch.rand(n, dtype=torch.float64, device="cuda")
    out = torch.empty(5, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert f(v.data_ptr(), v.data_ptr(), v.data_ptr(), n, 9.81, 0.4, 0.5, 0.5,
             out.data_ptr(), stream) == 0  # first call in this context
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(50):
        assert f(v.data_ptr(), v.data_ptr(), v.data_ptr(), n, 9.81, 0.4, 0.5, 0.5,
                 out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    host = v.cpu().numpy()
    assert tuple(out.cpu().numpy()) == _host_dt(host, host, host, 9.81, 0.4, 0.5, 0.5)


def test_cfl_dt_noalloc_rejects_bad_sizes(cuda_lib):
    import torch
    f = _bind(cuda_lib)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert f(p, p, p, 0, 9.81, 0.4, 1.0, 1.0, p, None) == -1          # DAMPM_ERR_ARG
    assert f(p, p, p, 1 << 31, 9.81, 0.4, 1.0, 1.0, p, None) == -4    # DAMPM_ERR_CAPACITY
    assert f(None, p, p, 4, 9.81, 0.4, 1.0, 1.0, p, None) == -1
    assert f(p, p, p, 4, 9.81, 0.4, 0.0, 1.0, p, None) == -1
