"""hosono_cfl_noalloc: the CFL step for callers that cannot allocate device
memory (inside a stream capture, under a foreign pool allocator, in loops that
must not enter the allocator).  It keeps its reduction scratch in a
file-scope device array instead of a cudaMalloc'd buffer; its dt must equal
the regular hosono_gpu_cfl's on the same state, call after call.

Named to be collected last: a failure here leaves every other test run.
"""
import ctypes

import pytest

import parfiles
import pkg


def _device_V(torch, V, pitch):
    """Copy a host V (nyTot, nxTot, 10) into a caller-owned device array in
    the library's SoA layout: 10 planes of nyTot rows, `pitch` doubles a row."""
    nyt, nxt, _ = V.shape
    dev = torch.zeros((10, nyt, pitch), dtype=torch.float64, device="cuda")
    dev[:, :, :nxt] = torch.from_numpy(V.transpose(2, 0, 1).copy()).cuda()
    return dev


def test_noalloc_rejects_grids_beyond_its_scratch():
    """ny beyond HOSONO_NOALLOC_MAX_ROWS is refused before any GPU work."""
    m = pkg.load()
    lib = m.load_library()
    ny = m.NOALLOC_MAX_ROWS + 1
    pitch = 64
    rc = lib.hosono_cfl_noalloc(ctypes.c_void_p(256), 32, ny, 4, pitch, pitch * (ny + 8), 0.1, 0.1, 0.8, 0,
                                ctypes.c_void_p(256), None)
    assert rc == m.EINVAL


@pytest.mark.gpu
def test_noalloc_cfl_equals_cfl_on_two_calls(tmp_par_dir):
    import torch

    m = pkg.load()
    lib = m.load_library()
    par = parfiles.make(tmp_par_dir, "noalloc_ot", parfiles.orszag_tang(96, 2))
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    p = s.params
    pitch = (s.nxt + 31) // 32 * 32
    plane = pitch * s.nyt
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        if call == 1:  # second call on a different state: one step later
            s.timeStep_advanceSolution(s.cfl_computedt())
        _, V, _ = s.download()
        V_dev = _device_V(torch, V, pitch)
        expected = s.cfl_computedt()
        dt_dev.fill_(-1.0)
        torch.cuda.synchronize()
        rc = lib.hosono_cfl_noalloc(ctypes.c_void_p(V_dev.data_ptr()), p.nx, p.ny, p.ngc, pitch, plane, p.dx, p.dy,
                                    p.cfl, p.force_hydro, ctypes.c_void_p(dt_dev.data_ptr()),
                                    ctypes.c_void_p(stream) if stream else None)
        assert rc == m.OK
        torch.cuda.synchronize()
        # the same arithmetic as hosono_gpu_cfl (strict build): equal bit for bit
        assert dt_dev.item() == expected, (call, dt_dev.item(), expected)
    s.close()
