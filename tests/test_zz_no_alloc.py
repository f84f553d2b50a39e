"""swpc_vmax_noalloc: the report maximum for callers that own their device
arrays and may not allocate.  Its result must equal swpc_vmax of a context
holding the same wavefield (both reduce the same cells with an exact max, so
the comparison is bitwise, inside the suite's 1e-5 bar).  The file name makes
pytest collect it last: the entry point shares one scratch array per device,
so it must also hold up after every other test has run in the process."""
import ctypes as C

import numpy as np
import pytest

from models import small3d
from openswpc_b200 import _lib
from openswpc_b200._lib import fptr
from openswpc_b200.swpc3d import Swpc3D


def _call(lib, vx, vy, vz, kob, p, uc, stream, ld_k=None, ld_i=None):
    out = np.full(3, -1.0, np.float32)
    rc = lib.swpc_vmax_noalloc(C.c_void_p(vx), C.c_void_p(vy), C.c_void_p(vz), C.c_void_p(kob), p.nx, p.ny, p.nz,
                               p.na, ld_k or p.nz + 6, ld_i or p.nx + 6, C.c_float(uc), C.c_void_p(stream), fptr(out))
    return rc, out


def test_noalloc_rejects_bad_sizes_before_touching_the_device():
    lib = _lib.load()
    p = small3d()
    fake = 16   # never dereferenced: every check below returns before any CUDA call
    assert _call(lib, 0, fake, fake, fake, p, 1.0, 0)[0] == _lib.SWPC_ERR_ARG
    assert _call(lib, fake, fake, fake, fake, p, 1.0, 0, ld_k=p.nz + 5)[0] == _lib.SWPC_ERR_ARG
    big = small3d(ny=_lib.SWPC_NOALLOC_MAX_NY + 1)
    rc, out = _call(lib, fake, fake, fake, fake, big, 1.0, 0)
    assert rc == _lib.SWPC_ERR_LIMIT
    assert (out == -1.0).all()


def _state(torch, p, nsteps, scale):
    """Run `nsteps` steps, optionally scale the velocities in place, and return
    (device copies of vx, vy, vz, kob, swpc_vmax of the context, UC)."""
    with Swpc3D(p) as sim:
        sim.run(1, nsteps)
        if scale != 1.0:
            for f in (_lib.F_VX, _lib.F_VY, _lib.F_VZ):
                sim.upload(f, sim.download(f) * np.float32(scale))
        ref = sim.kernel__vmax()
        dev = [torch.from_numpy(sim.download(f)).cuda() for f in (_lib.F_VX, _lib.F_VY, _lib.F_VZ)]
        dev.append(torch.from_numpy(np.ascontiguousarray(sim.medium.kob, np.int32)).cuda())
        return dev, ref, float(sim.UC)


@pytest.mark.gpu
def test_noalloc_vmax_matches_context_vmax_on_calls_in_a_row():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    pa = small3d(nt=60)
    pb = small3d(nx=32, ny=28, nz=24, na=6, nt=40)
    # b has fewer rows and maxima 1000x smaller: a stale row or result word
    # left by the call on a would show in b's result
    da, ra, uca = _state(torch, pa, 40, 1.0)
    db, rb, ucb = _state(torch, pb, 30, 1e-3)
    assert (ra > 0).all() and (rb > 0).all() and (rb < ra).all()
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    orders = [((pa, da, ra, uca), (pb, db, rb, ucb)), ((pb, db, rb, ucb), (pa, da, ra, uca))]
    for n, order in enumerate(orders):
        free0 = torch.cuda.mem_get_info()[0]
        for p, d, ref, uc in order:
            rc, out = _call(lib, *[t.data_ptr() for t in d], p, uc, stream)
            assert rc == _lib.SWPC_OK
            np.testing.assert_allclose(out, ref, rtol=1e-5, atol=0)
            assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
        # once the library's device code is loaded (first call), the calls
        # allocate nothing on the device
        if n > 0:
            assert torch.cuda.mem_get_info()[0] == free0


@pytest.mark.gpu
def test_noalloc_vmax_reports_divergence():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    p = small3d(nt=20)
    d, ref, uc = _state(torch, p, 10, 1.0)
    # a spike at a reduced cell (k = kob + 1 of column i = j = 20)
    i = j = 20
    k = int(d[3][j + 2, i + 2].item()) + 1
    d[2][j + 2, i + 2, k + 2] = 1e25
    rc, out = _call(lib, *[t.data_ptr() for t in d], p, uc, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.SWPC_ERR_DIVERGED
    assert out[2] == np.float32(1e25) and out[0] == ref[0] and out[1] == ref[1]
