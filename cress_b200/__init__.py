"""cress_b200: B200 (sm_100a) implementation of CReSS's solver time integration.

This module is the host-side mirror of the reference's call interface
(the Fortran module procedures s_smalldrv, s_hevi, ... of SrcOrig/), bound
through ctypes to the C-ABI library built from cress_b200/csrc
(declarations: include/cress_b200.h).  Arrays cross the boundary as
float32 numpy arrays in the reference layout a(0:ni+1, 0:nj+1, 1:nk), i.e.
numpy shape (nk, nj+2, ni+2) in C order (x fastest).

There is no CPU fallback: if the shared library is missing or cannot be
loaded, every call raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcress_b200.so")

# Field and level ids (include/cress_b200.h: enum cress_field / cress_level).
FIELDS = ["u", "v", "w", "pp", "ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng", "tke"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
PAST, NOW, FUTURE, FORCING = 0, 1, 2, 3
NTILES = 14   # HE-VI tile shapes (cress_cfg.tile)
# enum cress_base order
BASE_NAMES = ["jcb", "jcb8u", "jcb8v", "jcb8w", "rbr", "ptbr", "rst", "rst8u", "rst8v",
              "rst8w", "rcsq"]

ERRORS = {1: "CRESS_E_ARG", 2: "CRESS_E_UNSUPPORTED", 3: "CRESS_E_CUDA",
          4: "CRESS_E_NONUNIFORM", 5: "CRESS_E_NONFINITE", 6: "CRESS_E_TIMEOUT",
          7: "CRESS_E_STATE"}


class CressError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Cfg(ctypes.Structure):
    """cress_cfg: resolved namelist values."""
    _fields_ = [("ni", ctypes.c_int), ("nj", ctypes.c_int), ("nk", ctypes.c_int),
                ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
                ("sthopt", ctypes.c_int), ("impopt", ctypes.c_int), ("divopt", ctypes.c_int),
                ("buyopt", ctypes.c_int), ("gwmopt", ctypes.c_int), ("weicoe", ctypes.c_float),
                ("wbc", ctypes.c_int), ("ebc", ctypes.c_int), ("sbc", ctypes.c_int),
                ("nbc", ctypes.c_int), ("bbc", ctypes.c_int), ("tbc", ctypes.c_int),
                ("tile", ctypes.c_int),
                ("advopt", ctypes.c_int), ("smtopt", ctypes.c_int), ("vspopt", ctypes.c_int),
                ("coropt", ctypes.c_int), ("tubopt", ctypes.c_int), ("cphopt", ctypes.c_int),
                ("smhcoe", ctypes.c_float), ("smvcoe", ctypes.c_float), ("filcoe", ctypes.c_float),
                ("fc", ctypes.c_float), ("vspvar", ctypes.c_char * 16),
                ("thresq", ctypes.c_float), ("gwave", ctypes.c_float), ("reserved", ctypes.c_int * 6)]


_lib = None
_FP = ctypes.POINTER(ctypes.c_float)


def lib():
    """Load the C-ABI library (raises if it is absent: no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing; run `python -m cress_b200.build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.cress_last_error.restype = ctypes.c_char_p
    L.cress_abi_version.restype = ctypes.c_int
    L.cress_create.argtypes = [ctypes.POINTER(Cfg), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.cress_destroy.argtypes = [ctypes.c_void_p]
    L.cress_destroy.restype = None
    L.cress_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.cress_sync.argtypes = [ctypes.c_void_p]
    L.cress_set_base3d.argtypes = [ctypes.c_void_p, ctypes.POINTER(_FP)]
    L.cress_put_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _FP]
    L.cress_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _FP]
    L.cress_small_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]
    L.cress_smalldrv.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float] + [_FP] * 12
    L.cress_launch_count.argtypes = [ctypes.c_void_p]
    L.cress_launch_count.restype = ctypes.c_longlong
    L.cress_set_base_large.argtypes = [ctypes.c_void_p, _FP, _FP, _FP, ctypes.c_int]
    L.cress_large_step.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_float, ctypes.c_int,
                                   ctypes.c_float]
    L.cress_set_base_moist.argtypes = [ctypes.c_void_p, _FP, _FP]
    L.cress_cloudphy.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_float]
    L.cress_satadjst.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]
    L.cress_get_precip.argtypes = [ctypes.c_void_p, _FP]
    L.cress_put_precip.argtypes = [ctypes.c_void_p, _FP]
    L.cress_get_phase.argtypes = [ctypes.c_void_p, ctypes.c_int, _FP]
    L.cress_put_phase.argtypes = [ctypes.c_void_p, ctypes.c_int, _FP]
    vp, i, ll, ull, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.c_float
    L.cress_mlp_param_count.restype = i
    L.cress_mlp_create.argtypes = [i, ull, ctypes.POINTER(vp)]
    L.cress_mlp_destroy.argtypes = [vp]
    L.cress_mlp_destroy.restype = None
    for name in ("cress_mlp_get_params", "cress_mlp_set_params", "cress_mlp_get_norm", "cress_mlp_set_norm"):
        getattr(L, name).argtypes = [vp, _FP]
    L.cress_mlp_forward.argtypes = [vp, i, _FP, _FP]
    L.cress_mlp_loss_grad.argtypes = [vp, i, _FP, _FP, _FP, _FP]
    L.cress_mlp_reserve.argtypes = [vp, ll]
    L.cress_mlp_add_tuples.argtypes = [vp, ll, _FP, _FP]
    L.cress_mlp_get_tuples.argtypes = [vp, ll, ll, _FP, _FP]
    L.cress_mlp_tuple_count.argtypes = [vp]
    L.cress_mlp_tuple_count.restype = ll
    L.cress_mlp_fit_norm.argtypes = [vp]
    L.cress_mlp_train.argtypes = [vp, i, i, f, ull, _FP]
    L.cress_set_learned_micro.argtypes = [vp, vp, i, f]
    L.cress_learned_stats.argtypes = [vp, ctypes.POINTER(ll), ctypes.POINTER(ll)]
    L.cress_set_tuple_sampling.argtypes = [vp, vp, i, f, ull]
    L.cress_set_graphs.argtypes = [vp, i]
    L.cress_diagnostics.argtypes = [vp, i, ctypes.POINTER(ctypes.c_double)]
    L.cress_ensemble_create.argtypes = [ctypes.POINTER(vp), i, ctypes.POINTER(vp)]
    L.cress_ensemble_destroy.argtypes = [vp]
    L.cress_ensemble_destroy.restype = None
    L.cress_ensemble_large_step.argtypes = [vp, ll, f, i, f]
    L.cress_ensemble_set_graphs.argtypes = [vp, i]
    L.cress_ensemble_set_tile.argtypes = [vp, i]
    L.cress_ensemble_autotune.argtypes = [vp, i, f, i, ctypes.POINTER(i), ctypes.POINTER(f)]
    L.cress_autotune.argtypes = [vp, i, f, i, ctypes.POINTER(i), ctypes.POINTER(f)]
    L.cress_set_spin_limit.argtypes = [vp, i]
    L.cress_get_fields_async.argtypes = [vp, i, i, ctypes.POINTER(i), ctypes.POINTER(_FP)]
    L.cress_wait_fields.argtypes = [vp]
    L.cress_wait_fields_to.argtypes = [vp, i]
    L.cress_put_fields_async.argtypes = [vp, i, i, ctypes.POINTER(i), ctypes.POINTER(_FP)]
    ll = ctypes.c_longlong
    L.cress_dump_3d.argtypes = [vp, i, ctypes.c_char_p, vp, ll, ctypes.POINTER(ll), ctypes.c_char_p, i]
    L.cress_restart_write.argtypes = [vp, vp, ll, ctypes.POINTER(ll)]
    L.cress_restart_read.argtypes = [vp, vp, ll]
    L.cress_slab_group_create.argtypes = [i, ctypes.POINTER(vp)]
    L.cress_slab_group_destroy.argtypes = [vp]
    L.cress_slab_group_destroy.restype = None
    L.cress_slab_group_set_timeout.argtypes = [vp, i]
    L.cress_slab_attach_local.argtypes = [vp, vp, i]
    L.cress_slab_nccl_id.argtypes = [vp]
    L.cress_slab_attach_nccl.argtypes = [vp, i, i, vp]
    L.cress_slab_detach.argtypes = [vp]
    dp = ctypes.POINTER(ctypes.c_double)
    L.cress_base_state.argtypes = [i, dp, dp, i, dp, i, i, ctypes.c_double, ctypes.c_double, dp, i]
    _lib = L
    return L


def _check(code):
    if code != 0:
        raise CressError(code, lib().cress_last_error().decode())


def fptr(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


BASE_COLUMNS = ["ubr", "vbr", "pbr", "ptbr", "qvbr", "rbr", "ptvbr", "pibr", "rst", "rst8w", "rcsq"]


def base_state(nk, zph, jcb, z, u, v, pt, qv, psnd0, thresq=1e-12, tvar="p", hvar="r", device=0):
    """The base state from a height-level sounding, computed on the device
    in FP64 (cress_base_state): a dict of BASE_COLUMNS, each an array of
    nk+1 doubles by level index k.  zph, jcb: the column's w-level heights
    and Jacobian by index k; the sounding arrays are its levels 1..nlev."""
    dp = ctypes.POINTER(ctypes.c_double)
    zph = np.ascontiguousarray(zph, np.float64)
    jcb = np.ascontiguousarray(jcb, np.float64)
    assert zph.size == nk + 1 and jcb.size == nk + 1
    snd = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in (z, u, v, pt, qv)]))
    out = np.zeros((len(BASE_COLUMNS), nk + 1))
    _check(lib().cress_base_state(int(nk), zph.ctypes.data_as(dp), jcb.ctypes.data_as(dp), len(z),
                                  snd.ctypes.data_as(dp), ord(tvar), ord(hvar), float(psnd0), float(thresq),
                                  out.ctypes.data_as(dp), int(device)))
    return dict(zip(BASE_COLUMNS, out))


class SlabGroup:
    """The ranks of a y-slab decomposition that live in this process
    (cress_slab_group): each rank's Solver attaches with slab_attach and is
    stepped by its own thread."""

    def __init__(self, nranks, timeout_ms=None):
        h = ctypes.c_void_p()
        _check(lib().cress_slab_group_create(int(nranks), ctypes.byref(h)))
        self._h = h
        if timeout_ms is not None:
            _check(lib().cress_slab_group_set_timeout(h, int(timeout_ms)))

    def close(self):
        if getattr(self, "_h", None):
            lib().cress_slab_group_destroy(self._h)
            self._h = None


def slab_nccl_id():
    """128 bytes naming a new NCCL communicator (cress_slab_nccl_id)."""
    b = ctypes.create_string_buffer(128)
    _check(lib().cress_slab_nccl_id(b))
    return b.raw


class Solver:
    """One domain on one GPU (a cress_ctx)."""

    def __init__(self, ni, nj, nk, dx, dy, dz, sthopt=0, divopt=2, buyopt=1, weicoe=0.6, impopt=1,
                 tile=0, device=0, smtopt=3, smhcoe=0.001, smvcoe=0.0004, vspopt=2,
                 vspvar="oooxoooooo", coropt=0, fc=0.0, filcoe=0.1, cphopt=0, thresq=1e-12,
                 tubopt=0, obc=0, gwave=20.0, advopt=2):
        L = lib()
        c = Cfg()
        c.ni, c.nj, c.nk = ni, nj, nk
        c.dx, c.dy, c.dz = dx, dy, dz
        c.sthopt, c.impopt, c.divopt, c.buyopt, c.gwmopt = sthopt, impopt, divopt, buyopt, 0
        c.weicoe = weicoe
        # obc 0: periodic on all sides; 4, 5, 7: open radiation x boundaries
        c.wbc = c.ebc = obc if obc else -1
        c.sbc = c.nbc = -1
        c.gwave = gwave
        c.bbc = c.tbc = 2
        c.tile = tile
        c.advopt, c.smtopt, c.vspopt, c.coropt, c.tubopt, c.cphopt = advopt, smtopt, vspopt, coropt, tubopt, cphopt
        c.smhcoe, c.smvcoe, c.filcoe, c.fc = smhcoe, smvcoe, filcoe, fc
        c.vspvar = vspvar.encode()[:15]
        c.thresq = thresq
        self.cfg = c
        self.shape = (nk, nj + 2, ni + 2)
        h = ctypes.c_void_p()
        _check(L.cress_create(ctypes.byref(c), device, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().cress_destroy(self._h)
            self._h = None

    __del__ = close

    def set_stream(self, stream_ptr):
        _check(lib().cress_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def sync(self):
        _check(lib().cress_sync(self._h))

    def set_spin_limit(self, probes):
        """Failure-path test hook: probes per HE-VI ring wait before it gives
        up (0: at once; negative: the default)."""
        _check(lib().cress_set_spin_limit(self._h, int(probes)))

    def set_base3d(self, base):
        arrs = [np.ascontiguousarray(base[n], dtype=np.float32) for n in BASE_NAMES]
        for a in arrs:
            assert a.shape == self.shape, (a.shape, self.shape)
        ptrs = (_FP * len(arrs))(*[fptr(a) for a in arrs])
        _check(lib().cress_set_base3d(self._h, ptrs))

    def put_field(self, name, level, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32)
        assert a.shape == self.shape
        _check(lib().cress_put_field(self._h, FIELD_ID[name], level, fptr(a)))

    def get_field(self, name, level, out=None):
        a = np.empty(self.shape, np.float32) if out is None else out
        assert a.shape == self.shape and a.dtype == np.float32 and a.flags.c_contiguous
        _check(lib().cress_get_field(self._h, FIELD_ID[name], level, fptr(a)))
        return a

    def get_fields_async(self, level, names, outs):
        """Start copying fields of one level into host arrays (see
        cress_get_fields_async); they are filled after wait_fields().  The
        arrays must stay alive (and preferably be page-locked) until then."""
        for a in outs:
            assert a.shape == self.shape and a.dtype == np.float32 and a.flags.c_contiguous
        ids = (ctypes.c_int * len(names))(*[FIELD_ID[n] for n in names])
        ptrs = (_FP * len(outs))(*[fptr(a) for a in outs])
        # two read-backs may be in flight: keep both sets of arguments alive
        self._async_keep = (getattr(self, "_async_keep", ()) + ((ids, ptrs, list(outs)),))[-2:]
        _check(lib().cress_get_fields_async(self._h, int(level), len(names), ids, ptrs))

    def wait_fields(self, in_flight=0):
        """Wait until at most `in_flight` (0 or 1) read-backs are running."""
        _check(lib().cress_wait_fields_to(self._h, int(in_flight)))

    def put_fields_async(self, level, names, arrs):
        """Start copying host arrays into fields of one level (see
        cress_put_fields_async): the copies overlap the work already queued
        and the values are in the level for the calls that follow.  The
        arrays (float32, C-contiguous, preferably page-locked) are kept
        referenced here and must not change until a synchronizing call."""
        for a in arrs:
            assert a.shape == self.shape and a.dtype == np.float32 and a.flags.c_contiguous
        ids = (ctypes.c_int * len(names))(*[FIELD_ID[n] for n in names])
        ptrs = (_FP * len(arrs))(*[fptr(a) for a in arrs])
        if not hasattr(self, "_put_keep"):
            self._put_keep = {}
        self._put_keep[int(level)] = (ids, ptrs, list(arrs))
        _check(lib().cress_put_fields_async(self._h, int(level), len(names), ids, ptrs))

    def dump_3d(self, dmpvar, level=NOW, out=None):
        """The 3-D dump records of one level as s_outdmp writes them (dmplev
        = 1, dmpfmt = 2; see cress_dump_3d): returns (records, names) with
        records a float32 array (nvar, nz, ny, nx) whose bytes are the .bin
        file, names the dumped variables in file order.  out: an array of
        that shape to fill (e.g. page-locked memory)."""
        L = lib()
        n = ctypes.c_longlong()
        names = ctypes.create_string_buffer(512)
        _check(L.cress_dump_3d(self._h, int(level), dmpvar.encode(), None, 0, ctypes.byref(n), names, 512))
        vs = [v for v in names.value.decode().split(",") if v]
        nk, nj2, ni2 = self.shape
        shape = (len(vs), nk - 3, nj2 - 5, ni2 - 5)
        if out is None:
            out = np.empty(shape, np.float32)
        assert out.shape == shape and out.dtype == np.float32 and out.flags.c_contiguous
        if vs:
            _check(L.cress_dump_3d(self._h, int(level), dmpvar.encode(), out.ctypes.data_as(ctypes.c_void_p),
                                   out.nbytes, ctypes.byref(n), None, 0))
        assert n.value == out.nbytes
        return out, vs

    def restart_size(self):
        n = ctypes.c_longlong()
        _check(lib().cress_restart_write(self._h, None, 0, ctypes.byref(n)))
        return n.value

    def restart_write(self, out=None):
        """The device-held restart records (cress_restart_write) as bytes
        (a uint8 array; out: one of restart_size() bytes to fill)."""
        L = lib()
        n = ctypes.c_longlong()
        if out is None:
            out = np.empty(self.restart_size(), np.uint8)
        assert out.dtype == np.uint8 and out.flags.c_contiguous
        _check(L.cress_restart_write(self._h, out.ctypes.data_as(ctypes.c_void_p), out.nbytes, ctypes.byref(n)))
        return out

    def restart_read(self, data):
        """Restore the device state from restart records (cress_restart_read)."""
        a = np.ascontiguousarray(np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data,
                                 np.uint8)
        _check(lib().cress_restart_read(self._h, a.ctypes.data_as(ctypes.c_void_p), a.nbytes))

    def slab_attach(self, group, rank):
        """Make this context rank `rank` of a y-slab decomposition whose ranks
        are contexts of this process (cress_slab_attach_local)."""
        _check(lib().cress_slab_attach_local(self._h, group._h, int(rank)))
        self._slab_group = group

    def slab_attach_nccl(self, rank, nranks, uid):
        """Rank `rank` of `nranks` processes exchanging over NCCL; uid: the
        128 bytes of slab_nccl_id() from one rank."""
        b = ctypes.create_string_buffer(bytes(uid), 128)
        _check(lib().cress_slab_attach_nccl(self._h, int(rank), int(nranks), b))

    def slab_detach(self):
        _check(lib().cress_slab_detach(self._h))
        self._slab_group = None

    def small_steps(self, nsstp, dts):
        _check(lib().cress_small_steps(self._h, int(nsstp), float(dts)))

    def smalldrv(self, nsstp, dts, up, vp, wp, ppp, ufrc, vfrc, wfrc, pfrc, out=None):
        """s_smalldrv with host arrays (SrcOrig/smalldrv.f90:343-398)."""
        ins = [np.ascontiguousarray(a, dtype=np.float32) for a in
               (up, vp, wp, ppp, ufrc, vfrc, wfrc, pfrc)]
        outs = out if out is not None else [np.empty(self.shape, np.float32) for _ in range(4)]
        _check(lib().cress_smalldrv(self._h, int(nsstp), float(dts),
                                    *[fptr(a) for a in ins], *[fptr(a) for a in outs]))
        return outs

    def launch_count(self):
        return lib().cress_launch_count(self._h)

    def set_base_large(self, ubr, vbr, rbct, ksp0):
        """Base winds and the Rayleigh coefficient rbct(:,:,:,2) (SrcOrig/vspdmp.f90)."""
        arrs = [np.ascontiguousarray(x, dtype=np.float32) for x in (ubr, vbr, rbct)]
        for a in arrs:
            assert a.shape == self.shape
        _check(lib().cress_set_base_large(self._h, *[fptr(a) for a in arrs], int(ksp0)))

    def large_step(self, ctime, dtb, nsstp, dts):
        """One s_intgdrv leapfrog step on the device-resident state.  ctime is
        the model time of the present level in ms (0: first step, no
        Asselin filter); dtb, dts are that step's large and small steps."""
        _check(lib().cress_large_step(self._h, int(ctime), float(dtb), int(nsstp), float(dts)))

    def set_base_moist(self, pbr, qvbr):
        arrs = [np.ascontiguousarray(x, dtype=np.float32) for x in (pbr, qvbr)]
        _check(lib().cress_set_base_moist(self._h, *[fptr(a) for a in arrs]))

    def cloudphy(self, dtb, thresq=1e-12):
        """s_cloudphy (cphopt=3) on the device-resident past and future levels."""
        _check(lib().cress_cloudphy(self._h, float(dtb), float(thresq)))

    def satadjst(self, level, thresq=1e-12):
        _check(lib().cress_satadjst(self._h, int(level), float(thresq)))

    def set_graphs(self, on=True):
        """Replay whole large steps from CUDA graphs."""
        _check(lib().cress_set_graphs(self._h, int(bool(on))))

    def set_learned_micro(self, mlp, chunk=0, resid_tol=0.5):
        """Use `mlp` (an Mlp) for the process rates of s_cloudphy; None
        returns to the plain scheme."""
        _check(lib().cress_set_learned_micro(self._h, mlp._h if mlp else None, int(chunk), float(resid_tol)))
        self._mlp = mlp

    def learned_stats(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().cress_learned_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_tuple_sampling(self, mlp, stride=64, keep_zero=0.1, seed=1):
        _check(lib().cress_set_tuple_sampling(self._h, mlp._h if mlp else None, int(stride),
                                              float(keep_zero), int(seed)))
        self._sampler = mlp

    DIAG_NAMES = ("water", "precip", "mass", "max_u", "max_v", "max_w", "max_ptp", "nonfinite")

    def diagnostics(self, level=NOW, check=True):
        """FP64 domain sums and maxima of one time level as a dict (see
        cress_diagnostics); with check=True a non-finite value raises
        CressError (CRESS_E_NONFINITE)."""
        out = (ctypes.c_double * 8)()
        rc = lib().cress_diagnostics(self._h, int(level), out)
        if check or rc != 5:
            _check(rc)
        return dict(zip(self.DIAG_NAMES, list(out)))

    def autotune(self, nsstp=10, dts=1.0, reps=3):
        """Time every HE-VI tile shape on the current state and keep the
        fastest; returns (best tile, milliseconds per substep per tile,
        -1 for shapes the grid cannot use)."""
        best = ctypes.c_int(-1)
        ms = (ctypes.c_float * NTILES)()
        _check(lib().cress_autotune(self._h, int(nsstp), float(dts), int(reps), ctypes.byref(best), ms))
        return best.value, list(ms)

    def get_precip(self):
        ni, nj = self.shape[2] - 2, self.shape[1] - 2
        a = np.empty((5, 2, nj + 2, ni + 2), np.float32)
        _check(lib().cress_get_precip(self._h, fptr(a)))
        return a

    def put_precip(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(lib().cress_put_precip(self._h, fptr(a)))

    def get_phase(self, name):
        """Open x: phase speeds of one field as ucpx(1:nj,1:nk,1:2), returned
        in C order with shape (2, nk, nj) (side, k, j)."""
        nk, nj = self.shape[0], self.shape[1] - 2
        a = np.empty((2, nk, nj), np.float32)
        _check(lib().cress_get_phase(self._h, FIELD_ID[name], fptr(a)))
        return a

    def put_phase(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(lib().cress_put_phase(self._h, FIELD_ID[name], fptr(a)))


class Ensemble:
    """Independent domains (Solver objects, any sizes) stepped together: each
    large step runs every member as Solver.large_step would, with the
    acoustic substeps of all members in one launch per substep (see the
    ensemble section of include/cress_b200.h).  Each member keeps its own
    stream; repeated steps replay one CUDA graph of the whole ensemble step
    unless graphs=False.  Close the ensemble before the members."""

    def __init__(self, members, graphs=True):
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m._h for m in self.members])
        h = ctypes.c_void_p()
        _check(lib().cress_ensemble_create(arr, len(self.members), ctypes.byref(h)))
        self._h = h
        if not graphs:
            _check(lib().cress_ensemble_set_graphs(self._h, 0))

    def sync(self):
        for m in self.members:
            m.sync()

    def large_step(self, ctime, dtb, nsstp, dts):
        _check(lib().cress_ensemble_large_step(self._h, int(ctime), float(dtb), int(nsstp), float(dts)))

    def set_tile(self, tile):
        """The batched acoustic kernel: 0 or 13 (see cress_ensemble_set_tile)."""
        _check(lib().cress_ensemble_set_tile(self._h, int(tile)))

    def autotune(self, nsstp, dts, reps=3):
        """Time the batched substep with tiles 0 and 13, keep the faster;
        returns (tile, {tile: ms per substep})."""
        best = ctypes.c_int(-1)
        ms = (ctypes.c_float * 2)()
        _check(lib().cress_ensemble_autotune(self._h, int(nsstp), float(dts), int(reps), ctypes.byref(best), ms))
        return best.value, {0: ms[0], 13: ms[1]}

    def close(self):
        if self._h:
            lib().cress_ensemble_destroy(self._h)
            self._h = None


class Mlp:
    """The learned-microphysics network on one device (see the cress_mlp_*
    section of include/cress_b200.h for inputs, outputs and layouts)."""

    NORM = 82
    N_IN, N_OUT = 16, 9

    def __init__(self, device=0, seed=1):
        h = ctypes.c_void_p()
        _check(lib().cress_mlp_create(int(device), int(seed), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().cress_mlp_destroy(self._h)
            self._h = None

    __del__ = close

    @staticmethod
    def param_count():
        return lib().cress_mlp_param_count()

    def get_params(self):
        a = np.empty(self.param_count(), np.float32)
        _check(lib().cress_mlp_get_params(self._h, fptr(a)))
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, np.float32)
        assert a.size == self.param_count()
        _check(lib().cress_mlp_set_params(self._h, fptr(a)))

    def get_norm(self):
        a = np.empty(self.NORM, np.float32)
        _check(lib().cress_mlp_get_norm(self._h, fptr(a)))
        return a

    def set_norm(self, a):
        a = np.ascontiguousarray(a, np.float32)
        assert a.size == self.NORM
        _check(lib().cress_mlp_set_norm(self._h, fptr(a)))

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((x.shape[0], self.N_OUT), np.float32)
        _check(lib().cress_mlp_forward(self._h, int(x.shape[0]), fptr(x), fptr(y)))
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = np.zeros(1, np.float32)
        g = np.empty(self.param_count(), np.float32)
        _check(lib().cress_mlp_loss_grad(self._h, int(x.shape[0]), fptr(x), fptr(t), fptr(loss), fptr(g)))
        return float(loss[0]), g

    def reserve(self, cap):
        _check(lib().cress_mlp_reserve(self._h, int(cap)))

    def add_tuples(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        _check(lib().cress_mlp_add_tuples(self._h, int(x.shape[0]), fptr(x), fptr(t)))

    def get_tuples(self, first=0, n=None):
        if n is None:
            n = self.tuple_count() - first
        x = np.empty((n, self.N_IN), np.float32)
        t = np.empty((n, self.N_OUT), np.float32)
        _check(lib().cress_mlp_get_tuples(self._h, int(first), int(n), fptr(x), fptr(t)))
        return x, t

    def tuple_count(self):
        return lib().cress_mlp_tuple_count(self._h)

    def fit_norm(self):
        _check(lib().cress_mlp_fit_norm(self._h))

    def train(self, steps, batch=8192, lr=1e-3, seed=1):
        losses = np.empty(max(int(steps), 1), np.float32)
        _check(lib().cress_mlp_train(self._h, int(steps), int(batch), float(lr), int(seed), fptr(losses)))
        return losses[:steps]
