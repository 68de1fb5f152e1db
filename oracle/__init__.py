"""CPU oracle for the CReSS hot path — TEST INFRASTRUCTURE ONLY.

A C++ restatement of the reference's Fortran routines (each function in
oracle/*.h cites the SrcOrig file:line it follows), compiled with g++
(-O2 -ffp-contract=off, no fast-math) into oracle/_build/liboracle_cress.so.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
it, always as the checker or the timed CPU baseline; the product library
(cress_b200) never imports, links or calls anything here.

Parity status: the reference is Fortran with no compiler in this image and
ships no golden outputs, so this restatement is pinned by the reference's
own formulas and by self-consistency checks (tests/test_oracle.py), not by
reference-produced vectors: parity unpinned.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle_cress.so")
LIB_OMP = os.path.join(BUILD, "liboracle_cress_omp.so")
SOURCES = ["oracle_capi.cpp", "oracle_dry.cpp", "oracle_moist.cpp"]
HEADERS = [f for f in os.listdir(HERE) if f.endswith(".h")]

_FP = ctypes.POINTER(ctypes.c_float)


def build(force=False):
    """Compile the oracle (plain and OpenMP builds) if sources changed."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    newest = max(os.path.getmtime(os.path.join(HERE, f)) for f in SOURCES + HEADERS)
    for out, extra in ((LIB, []), (LIB_OMP, ["-fopenmp", "-DORACLE_OMP=1"])):
        if not force and os.path.exists(out) and os.path.getmtime(out) >= newest:
            continue
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
               "-shared", "-o", out + ".tmp"] + extra + srcs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stderr)
        os.replace(out + ".tmp", out)
    return LIB


_libs = {}


def lib(omp=False):
    path = LIB_OMP if omp else LIB
    if path not in _libs:
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_small_steps.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
            ctypes.c_double, ctypes.c_int, ctypes.POINTER(_FP), ctypes.POINTER(_FP),
            ctypes.POINTER(_FP)]
        _libs[path] = L
    return _libs[path]


BASE_NAMES = ["jcb", "jcb8u", "jcb8v", "jcb8w", "rbr", "ptbr", "rst", "rst8u", "rst8v",
              "rst8w", "rcsq"]
DRY_BASE_NAMES = BASE_NAMES + ["ubr", "vbr"]
STATE_NAMES = ["u", "v", "w", "pp", "ptp"]


def vspdmp(nk, zph, vspbar, botbar):
    """Rayleigh coefficient rbct(k) (index k) and ksp0 of s_vspdmp, vspopt=2."""
    L = lib()
    L.oracle_vspdmp.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                ctypes.c_double, _FP]
    z = np.ascontiguousarray(zph, np.float64)
    r = np.zeros(nk + 1, np.float32)
    ksp0 = L.oracle_vspdmp(nk, z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), vspbar, botbar,
                           r.ctypes.data_as(_FP))
    return r, ksp0


def dry_steps(cfg, base, zph, past, now, nsteps, dtbig, dtsml, start=True, prec=32, fp64_solve=1,
              omp=False):
    """Run nsteps dry large steps (s_intgdrv) on the CPU; past/now are lists of
    u, v, w, pp, ptp arrays (and tke last with tubopt=2), updated in place.
    omp=True uses the OpenMP build."""
    L = lib(omp)
    L.oracle_dry_steps.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(_FP), ctypes.POINTER(_FP), ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int]
    io = (ctypes.c_int * 14)(cfg["ni"], cfg["nj"], cfg["nk"], cfg.get("divopt", 2),
                             cfg.get("buyopt", 1), int(fp64_solve), cfg.get("sthopt", 0),
                             cfg.get("smtopt", 3), cfg.get("vspopt", 2), cfg.get("coropt", 0),
                             cfg.get("tubopt", 0), cfg.get("impopt", 1), cfg.get("obc", 0),
                             cfg.get("advopt", 2))
    ro = (ctypes.c_double * 11)(cfg["dx"], cfg["dy"], cfg["dz"], cfg.get("weicoe", 0.6),
                                cfg.get("smhcoe", 0.001), cfg.get("smvcoe", 0.0004),
                                cfg.get("filcoe", 0.1), cfg.get("vspbar", 0.0),
                                cfg.get("botbar", 1e9), cfg.get("fc", 0.0), cfg.get("gwave", 20.0))
    z = np.ascontiguousarray(zph, np.float64)
    b = [np.ascontiguousarray(base[n], np.float32) for n in DRY_BASE_NAMES]
    st = list(past) + list(now)
    assert len(st) == (12 if cfg.get("tubopt", 0) == 2 else 10)
    for s in st:
        assert s.dtype == np.float32 and s.flags.c_contiguous
    rc = L.oracle_dry_steps(prec, io, ro, z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            (_FP * len(b))(*[_fp(x) for x in b]),
                            (_FP * len(st))(*[_fp(x) for x in st]), int(nsteps), float(dtbig),
                            float(dtsml), int(bool(start)))
    if rc != 0:
        raise RuntimeError(f"oracle_dry_steps failed ({rc})")


MOIST_BASE_NAMES = DRY_BASE_NAMES + ["pbr", "qvbr"]
MOIST_STATE_NAMES = STATE_NAMES + ["qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def moist_steps(cfg, base, zph, past, now, prec, nsteps, dtbig, dtsml, start=True, prec_bits=32,
                fp64_solve=1, omp=False):
    """Run nsteps moist (cphopt=3) large steps on the CPU.  past/now: lists of
    14 arrays in MOIST_STATE_NAMES order (15 with tke last when tubopt=2),
    updated in place; prec: the
    5 x 2 x (nj+2) x (ni+2) precipitation planes (in/out).  Returns npstp
    of the last step's sedimentation."""
    L = lib(omp)
    L.oracle_moist_steps.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(_FP), ctypes.POINTER(_FP), _FP, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int]
    io = (ctypes.c_int * 14)(cfg["ni"], cfg["nj"], cfg["nk"], cfg.get("divopt", 2),
                             cfg.get("buyopt", 1), int(fp64_solve), cfg.get("sthopt", 0),
                             cfg.get("smtopt", 3), cfg.get("vspopt", 2), cfg.get("coropt", 0),
                             cfg.get("tubopt", 0), cfg.get("impopt", 1), cfg.get("obc", 0),
                             cfg.get("advopt", 2))
    ro = (ctypes.c_double * 12)(cfg["dx"], cfg["dy"], cfg["dz"], cfg.get("weicoe", 0.6),
                                cfg.get("smhcoe", 0.001), cfg.get("smvcoe", 0.0004),
                                cfg.get("filcoe", 0.1), cfg.get("vspbar", 0.0),
                                cfg.get("botbar", 1e9), cfg.get("fc", 0.0), cfg.get("thresq", 1e-12),
                                cfg.get("gwave", 20.0))
    z = np.ascontiguousarray(zph, np.float64)
    b = [np.ascontiguousarray(base[n], np.float32) for n in MOIST_BASE_NAMES]
    st = list(past) + list(now)
    assert len(st) == (30 if cfg.get("tubopt", 0) == 2 else 28)
    for s in st:
        assert s.dtype == np.float32 and s.flags.c_contiguous
    assert prec.dtype == np.float32 and prec.flags.c_contiguous
    rc = L.oracle_moist_steps(prec_bits, io, ro, z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              (_FP * len(b))(*[_fp(x) for x in b]),
                              (_FP * len(st))(*[_fp(x) for x in st]), _fp(prec), int(nsteps),
                              float(dtbig), float(dtsml), int(bool(start)))
    if rc < 0:
        raise RuntimeError(f"oracle_moist_steps failed ({rc})")
    return rc


BASE_STATE_FIELDS = ["ubr", "vbr", "pbr", "ptbr", "qvbr", "rbr", "ptvbr", "pibr", "rst", "rst8w", "rcsq"]


def base_state(nk, zph, jcb, z, u, v, pt, qv, psnd0, thresq=1e-12, tvar="p", hvar="r", prec=64):
    """Base-state columns (index k = 0..nk) from a height-level sounding
    (set1d, vextlow, intrpsnd, setbase/bcbase, baserho, sndwave; base.h):
    dict of BASE_STATE_FIELDS.  zph, jcb: w-level heights and Jacobian by
    index k; the sounding arrays are levels 1..nlev."""
    L = lib()
    L.oracle_base_state.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    dp = ctypes.POINTER(ctypes.c_double)
    zph = np.ascontiguousarray(zph, np.float64)
    jcb = np.ascontiguousarray(jcb, np.float64)
    snd = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in (z, u, v, pt, qv)]))
    nlev = len(z)
    out = np.zeros((11, nk + 1))
    rc = L.oracle_base_state(int(prec), int(nk), zph.ctypes.data_as(dp), jcb.ctypes.data_as(dp), nlev,
                             snd.ctypes.data_as(dp), ord(tvar), ord(hvar), float(psnd0), float(thresq),
                             out.ctypes.data_as(dp))
    if rc != 0:
        raise RuntimeError(f"oracle_base_state failed ({rc})")
    return dict(zip(BASE_STATE_FIELDS, out))


def _fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


MICRO_PAST = ["ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng", "pp"]
MICRO_FUT = ["ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]
MICRO_BASE = ["ptbr", "rbr", "pbr", "jcb", "rst"]


def cloudphy(dims, base, past, fut, prec, dtb, dz, thresq=1e-12, bits=32):
    """One s_cloudphy call (cphopt=3) on the CPU.  past/fut: dicts of 3-D
    float32 arrays (MICRO_PAST / MICRO_FUT); fut and prec (5 x 2 x (nj+2) x
    (ni+2) float32: prc, prr, pri, prs, prg rate/accumulation) are updated
    in place.  Returns npstp, the sedimentation sub-step count."""
    ni, nj, nk = dims
    L = lib()
    L.oracle_cloudphy.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [ctypes.POINTER(_FP)] * 3 + [_FP]
    b = [np.ascontiguousarray(base[n], np.float32) for n in MICRO_BASE]
    p = [np.ascontiguousarray(past[n], np.float32) for n in MICRO_PAST]
    for n in MICRO_FUT:
        assert fut[n].dtype == np.float32 and fut[n].flags.c_contiguous
    assert prec.dtype == np.float32 and prec.flags.c_contiguous and prec.size == 10 * (ni + 2) * (nj + 2)
    f = [fut[n] for n in MICRO_FUT]
    rc = L.oracle_cloudphy(bits, ni, nj, nk, float(dtb), float(dz), float(thresq),
                           (_FP * len(b))(*[_fp(x) for x in b]), (_FP * len(p))(*[_fp(x) for x in p]),
                           (_FP * len(f))(*[_fp(x) for x in f]), _fp(prec))
    if rc < 0:
        raise RuntimeError(f"oracle_cloudphy failed ({rc})")
    return rc


def satadjst(dims, ptbr, pbr, pp, st, thresq=1e-12):
    """s_satadjst (cphopt=3) in place on st = dict with ptp, qv, qc, qi, ni."""
    ni, nj, nk = dims
    L = lib()
    L.oracle_satadjst.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, _FP, _FP, _FP, ctypes.POINTER(_FP)]
    L.oracle_satadjst.restype = None
    s = [st[n] for n in ("ptp", "qv", "qc", "qi", "ni")]
    for a in s:
        assert a.dtype == np.float32 and a.flags.c_contiguous
    L.oracle_satadjst(ni, nj, nk, float(thresq), _fp(np.ascontiguousarray(ptbr, np.float32)),
                      _fp(np.ascontiguousarray(pbr, np.float32)), _fp(np.ascontiguousarray(pp, np.float32)),
                      (_FP * 5)(*[_fp(a) for a in s]))


def small_steps(cfg, base, frc, state, nsstp, dts, prec=32, fp64_solve=1, omp=False):
    """Run s_smalldrv's loop (phy2cnt + nsstp x s_hevi, or s_heve when
    cfg["impopt"] == 0) on the CPU.

    cfg: dict with ni,nj,nk,dx,dy,dz,sthopt,divopt,buyopt,weicoe[,impopt].
    base: dict of 3-D float32 arrays (BASE_NAMES); frc: [ufrc,vfrc,wfrc,pfrc];
    state: [uf,vf,wf,ppf] (updated in place).
    """
    io = (ctypes.c_int * 11)(cfg["ni"], cfg["nj"], cfg["nk"], cfg.get("divopt", 2),
                             cfg.get("buyopt", 1), 0, 1, 2, 2, int(fp64_solve), cfg.get("impopt", 1))
    ro = (ctypes.c_double * 4)(cfg["dx"], cfg["dy"], cfg["dz"], cfg.get("weicoe", 0.6))
    b = [np.ascontiguousarray(base[n], np.float32) for n in BASE_NAMES]
    f = [np.ascontiguousarray(x, np.float32) for x in frc]
    for s in state:
        assert s.dtype == np.float32 and s.flags.c_contiguous
    rc = lib(omp).oracle_small_steps(prec, cfg.get("sthopt", 0), io, ro, float(dts), int(nsstp),
                                     (_FP * len(b))(*[_fp(x) for x in b]),
                                     (_FP * 4)(*[_fp(x) for x in f]),
                                     (_FP * 4)(*[_fp(x) for x in state]))
    if rc != 0:
        raise RuntimeError(f"oracle_small_steps failed ({rc})")
    return state
