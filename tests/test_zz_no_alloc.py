"""The allocation-free plane-ring entry point, for callers that must not call
cudaMalloc (an application whose own allocator already holds the device
memory, a process under a device-memory quota, a loop that cannot afford
cudaMalloc's implicit synchronisation).

beam_gpu_plane_rings_noalloc works only on the caller's device buffers and a
fixed scratch array inside the library; its output must equal that of
beam_gpu_plane_rings on the same inputs, on two calls in a row (the second
call reuses the scratch array the first one filled). Kept in a file of its own
that runs last."""
import ctypes

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden_field

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative to the largest value of each array, as test_plane_rings_match_oracle


def _noalloc(L, NN, Nmax, Nr, r2c_dev, planes, rings, out_dev, stream=None):
    ip = ctypes.POINTER(ctypes.c_int)
    L.beam_gpu_plane_rings_noalloc.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_void_p, ip, ip,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.beam_gpu_plane_rings_noalloc.restype = ctypes.c_int
    p = np.ascontiguousarray(planes, dtype=np.int32)
    r = np.ascontiguousarray(rings, dtype=np.int32)
    return L.beam_gpu_plane_rings_noalloc(NN, Nmax, Nr, r2c_dev.data_ptr(), p.ctypes.data_as(ip),
                                          r.ctypes.data_as(ip), len(p), out_dev.data_ptr(), stream)


def test_noalloc_plane_rings_match_the_allocating_entry_point(beamlib):
    torch = pytest.importorskip("torch")
    name = "nn96_r20"
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    field = golden_field(name)
    ctx = beamlib.Context(0)
    plan = beamlib.Plan(ctx, NN, UL, LL, BW, Nmax=Nmax, Nr=Nr)
    L = beamlib.load()
    r2c_dev = torch.from_numpy(field).cuda()
    calls = [([0, 0, 1, 3, Nmax - 1, 7], [0, 1, 0, 5, Nr - 1, 12]),
             ([2, 9, 31, 0], [19, 3, 10, 4])]
    side = torch.cuda.Stream()
    # two calls in a row on the legacy default stream, then the first again on a stream of the caller's
    for planes, rings, stream in [(*calls[0], None), (*calls[1], None), (*calls[0], side)]:
        want = plan.plane_rings(field, planes, rings)
        out = torch.full((len(planes), NN, NN, 2), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = _noalloc(L, NN, Nmax, Nr, r2c_dev, planes, rings, out, None if stream is None else stream.cuda_stream)
        assert rc == 0, L.beam_gpu_last_error_detail()
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex128)[..., 0]
        for k in range(len(planes)):
            scale = max(np.max(np.abs(want[k])), 1e-300)
            assert np.max(np.abs(got[k] - want[k])) <= TOL * scale, (planes[k], rings[k])
    plan.close()
    ctx.close()


def test_noalloc_rejects_requests_beyond_its_limits(beamlib):
    torch = pytest.importorskip("torch")
    L = beamlib.load()
    NN, Nmax, Nr = 64, 16, 10
    r2c_dev = torch.zeros((NN, NN, NN + 2), dtype=torch.float64, device="cuda")
    out = torch.zeros((1, NN, NN, 2), dtype=torch.float64, device="cuda")
    too_many = 4097  # BEAM_NOALLOC_MAX_JOBS + 1
    assert _noalloc(L, NN, Nmax, Nr, r2c_dev, [0] * too_many, [0] * too_many, out) == beamlib.BEAM_EINVAL
    assert _noalloc(L, NN, Nmax, Nr, r2c_dev, [Nmax], [0], out) == beamlib.BEAM_EINVAL
    assert _noalloc(L, NN, Nmax, Nr, r2c_dev, [0], [Nr], out) == beamlib.BEAM_EINVAL
    # tables beyond the 2 MiB array: ring 9 of 10 at NN=2048 reaches |k| = 1024 (about 3.3M modes);
    # refused on the host before any copy or launch touches the small buffers
    small = torch.zeros(64, dtype=torch.float64, device="cuda")
    assert _noalloc(L, 2048, 1024, 10, small, [0], [9], small) == beamlib.BEAM_EINVAL
    assert "bytes of tables" in L.beam_gpu_last_error_detail().decode()
    torch.cuda.synchronize()


def test_noalloc_refuses_a_capturing_stream(beamlib):
    """The tables are staged from a host buffer that the next call rewrites, so
    a copy captured into a graph would replay stale tables: a capturing stream
    is refused with BEAM_EINVAL and nothing is queued on it."""
    torch = pytest.importorskip("torch")
    L = beamlib.load()
    NN, Nmax, Nr = 64, 16, 10
    r2c_dev = torch.zeros((NN, NN, NN + 2), dtype=torch.float64, device="cuda")
    out = torch.zeros((1, NN, NN, 2), dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        graph.capture_begin()
        try:
            out.zero_()  # something for the graph to hold
            rc = _noalloc(L, NN, Nmax, Nr, r2c_dev, [0], [1], out, side.cuda_stream)
        finally:
            graph.capture_end()
    assert rc == beamlib.BEAM_EINVAL
    assert "captured" in L.beam_gpu_last_error_detail().decode()
    # the refusal left the device usable: a plain call still works
    assert _noalloc(L, NN, Nmax, Nr, r2c_dev, [0], [1], out) == 0
    torch.cuda.synchronize()
    del graph
