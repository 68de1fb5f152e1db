"""The no-allocation HE-VI substep entry point agrees with the context API.

cress_hevi_substep_noalloc is for callers that cannot call cudaMalloc from
inside their time loop (a host model whose device arrays sit in a pool it
sized at start-up, or a framework whose caching allocator owns the device).
Here torch plays that caller: it owns every device buffer, and the entry
point is called through the C-ABI twice in a row (substep 1, then substep 2
from substep 1's output).  Each result must match cress_smalldrv with
nsstp = 1 and 2 within the tolerance of the other small-step tests.  This
file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 2e-5  # per substep, relative to the field's max magnitude


def test_noalloc_matches_context_api_two_calls(cress):
    import torch
    from cress_b200 import cases

    nx, ny, nz = 70, 45, 30
    dx, dz, dts = 1000.0, 250.0, 0.5
    (ni, nj, nk), base, st, frc = cases.acoustic_case(nx, ny, nz, dx, dz, seed=21, sthopt=1)

    # Reference results through the context API (allocating path).
    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1)
    s.set_base3d(base)
    ref1 = s.smalldrv(1, dts, *st, *frc)
    ref2 = s.smalldrv(2, dts, *st, *frc)
    s.close()

    # Caller-owned device buffers in the padded layout.
    px = (ni + 2 + 31) // 32 * 32
    dev = torch.device("cuda", 0)

    def to_dev(a):
        t = torch.zeros((nk, nj + 2, px), dtype=torch.float32, device=dev)
        t[:, :, :ni + 2] = torch.from_numpy(np.ascontiguousarray(a))
        return t

    old = [to_dev(a) for a in st]
    frc_d = [to_dev(a) for a in frc]
    new1 = [to_dev(a) for a in st]   # start as copies of the old level (smalldrv.f90:343-346)
    new2 = [to_dev(a) for a in st]

    L = cress.lib()
    fn = L.cress_hevi_substep_noalloc
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.POINTER(cress.Cfg), ctypes.c_float, ctypes.POINTER(cress._FP)] + [P] * 12 + [P]
    fn.restype = ctypes.c_int
    c = cress.Cfg()
    c.ni, c.nj, c.nk = ni, nj, nk
    c.dx, c.dy, c.dz = dx, dx, dz
    c.sthopt, c.impopt, c.divopt, c.buyopt, c.gwmopt = 1, 1, 2, 1, 0
    c.weicoe = 0.6
    c.wbc = c.ebc = c.sbc = c.nbc = -1
    c.bbc = c.tbc = 2
    barrs = [np.ascontiguousarray(base[n], dtype=np.float32) for n in cress.BASE_NAMES]
    bptr = (cress._FP * len(barrs))(*[cress.fptr(a) for a in barrs])
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(o, n):
        rc = fn(ctypes.byref(c), dts, bptr, *[P(t.data_ptr()) for t in o], *[P(t.data_ptr()) for t in frc_d],
                *[P(t.data_ptr()) for t in n], P(stream))
        assert rc == 0, L.cress_last_error().decode()

    call(old, new1)   # first call: also sets up the device scratch address
    call(new1, new2)  # second call in a row reuses the same scratch
    torch.cuda.synchronize()

    stag = {"u": "u", "v": "v", "w": "s", "pp": "s"}
    for outs, refs, nsub in ((new1, ref1, 1), (new2, ref2, 2)):
        for name, t, r in zip(("u", "v", "w", "pp"), outs, refs):
            g = t[:, :, :ni + 2].cpu().numpy()
            m = np.zeros(g.shape, bool)
            ih = ni if stag[name] == "u" else ni - 1
            jh = nj if stag[name] == "v" else nj - 1
            m[:, 1:jh + 1, 1:ih + 1] = True
            scale = float(np.abs(r[m]).max()) + 1e-30
            err = float(np.abs(g[m] - r[m]).max())
            assert np.isfinite(g[m]).all(), name
            assert err <= RTOL * (nsub + 1) * scale, (nsub, name, err, scale)


def test_noalloc_rejects_too_many_levels(cress):
    import torch
    L = cress.lib()
    fn = L.cress_hevi_substep_noalloc
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.POINTER(cress.Cfg), ctypes.c_float, ctypes.POINTER(cress._FP)] + [P] * 12 + [P]
    c = cress.Cfg()
    c.ni, c.nj, c.nk = 20, 20, 300
    c.dx, c.dy, c.dz = 1000.0, 1000.0, 100.0
    c.impopt, c.divopt, c.buyopt = 1, 2, 1
    c.weicoe = 0.6
    c.wbc = c.ebc = c.sbc = c.nbc = -1
    c.bbc = c.tbc = 2
    dummy = torch.zeros(64, device="cuda")
    host = np.zeros(8, np.float32)
    bptr = (cress._FP * len(cress.BASE_NAMES))(*[cress.fptr(host)] * len(cress.BASE_NAMES))
    ptrs = [P(dummy.data_ptr())] * 12
    rc = fn(ctypes.byref(c), 0.5, bptr, *ptrs, P(0))
    assert rc == 1  # CRESS_E_ARG
    assert b"256" in L.cress_last_error()
