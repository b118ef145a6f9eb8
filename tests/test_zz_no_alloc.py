"""Allocation-free residual norms (rdst_residual_norms_noalloc).

Some callers cannot allocate device memory: code running while a CUDA
stream is captured into a graph (cudaMalloc is not a capturable call),
hosts whose device memory is handed out by a pool allocator, and paths that
cannot pay cudaMalloc's implicit synchronisation.  This entry point keeps
its scratch in a fixed array inside the library.  The test calls it through
the C ABI on device buffers the test owns and checks it against the norms
the existing rdst_step report gives for the same residual, on two calls in
a row.  The file is named to be collected last."""
import ctypes

import numpy as np
import pytest

import rhodst_b200
from rhodst_b200 import cases

pytestmark = pytest.mark.gpu


def _fn():
    lib = rhodst_b200.load_library()
    f = lib.rdst_residual_norms_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.rdst_last_error.restype = ctypes.c_char_p
    lib.rdst_last_error.argtypes = [ctypes.c_void_p]
    return lib, f


def test_residual_norms_noalloc_matches_step_report():
    import torch
    lib, fn = _fn()
    case = cases.forward_step_c1()
    s = rhodst_b200.solver_for(case)
    R = s.residual()                     # R(W) of the current state
    rep = s.step(1)[0]                   # the step reports the norms of that same R
    expect = np.array([rep["res_mag"]] + list(rep["res_l2"]))
    N = case.mesh.n_cells
    dev = torch.device("cuda", 0)
    Rd = torch.tensor(R, dtype=torch.float64, device=dev).contiguous()
    Vd = torch.tensor(case.mesh.V, dtype=torch.float64, device=dev).contiguous()
    out = torch.zeros(6, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for scale in (1.0, 2.0):             # two calls in a row sharing the scratch
        x = (Rd * scale).contiguous()
        st = fn(N, x.data_ptr(), Vd.data_ptr(), out.data_ptr(), stream)
        assert st == 0, lib.rdst_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, expect * scale, rtol=1e-12, atol=0.0), (got, expect * scale)


def test_residual_norms_noalloc_rejects_oversize():
    import torch
    lib, fn = _fn()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    st = fn(1_048_577, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert st == 7                       # RDST_ERR_ARG, nothing launched
    assert b"exceeds the fixed scratch capacity" in lib.rdst_last_error(None)


def test_residual_norms_noalloc_rejects_host_memory():
    """Host buffers are refused on the host, before anything is launched."""
    lib, fn = _fn()
    host = np.zeros(64, dtype=np.float64)
    p = host.ctypes.data
    st = fn(4, p, p, p, None)
    assert st == 7                       # RDST_ERR_ARG
    assert b"must be device memory" in lib.rdst_last_error(None)


def test_residual_norms_noalloc_follows_the_buffers_device():
    """A context created on another GPU first leaves the library's runtime
    on that GPU; the call must still run on the GPU holding the buffers
    (device 0 here) and give the same norms as the step report."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    lib, fn = _fn()
    case = cases.forward_step_c1()
    other = rhodst_b200.Solver(case.mesh, case.bcs, dict(case.options, device=1))
    other.set_primitive(case.p, case.U, case.T)
    s = rhodst_b200.solver_for(case)
    R = s.residual()
    rep = s.step(1)[0]
    expect = np.array([rep["res_mag"]] + list(rep["res_l2"]))
    dev = torch.device("cuda", 0)
    Rd = torch.tensor(R, dtype=torch.float64, device=dev).contiguous()
    Vd = torch.tensor(case.mesh.V, dtype=torch.float64, device=dev).contiguous()
    out = torch.zeros(6, dtype=torch.float64, device=dev)
    other.residual()                     # the library's runtime is now on device 1
    st = fn(case.mesh.n_cells, Rd.data_ptr(), Vd.data_ptr(), out.data_ptr(),
            torch.cuda.current_stream(dev).cuda_stream)
    assert st == 0, lib.rdst_last_error(None)
    torch.cuda.synchronize(dev)
    assert np.allclose(out.cpu().numpy(), expect, rtol=1e-12, atol=0.0)
    # buffers split across two GPUs are refused before any launch
    V1 = Vd.to(torch.device("cuda", 1))
    st = fn(case.mesh.n_cells, Rd.data_ptr(), V1.data_ptr(), out.data_ptr(), None)
    assert st == 7 and b"different devices" in lib.rdst_last_error(None)
