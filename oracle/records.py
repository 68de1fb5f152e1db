"""Oracle: the dump and restart file records of the reference, restated in
numpy from the host arrays (reference layout (nk, nj+2, ni+2), x fastest).

TEST INFRASTRUCTURE ONLY: the checker of the device-side record writers
(cress_dump_3d, cress_restart_write/read); nothing in the product imports it.

* dump_3d: s_outdmp for dmplev = 1 (SrcOrig/outdmp.f90:380-870) calling
  s_outdmp3d with dmpfmt = 2 (SrcOrig/outdmp3d.f90:159-238): per variable
  the records k = 2..nk-2 of (i = 2..ni-2, j = 2..nj-2), 'oxx' / 'xox' /
  'xxo' averaging .5*(a + a(+1)) in float32, s_totals for '-' on p and pt
  (SrcOrig/totals.f90: sbr + sp).
* restart_records: the records of s_outres after the base state
  (SrcOrig/outres.f90:903-1289) for cphopt 0 or 3 (haiopt = 0), tubopt
  0/1/2, open x or periodic, each framed as a Fortran sequential
  unformatted record (4-byte length before and after the payload).
"""
import numpy as np

F32 = np.float32


def _avg(a, axis):
    """.5*(a + a(+1)) along axis 2 (x), 1 (y) or 0 (z) on the dump region."""
    sl = [slice(1, a.shape[0] - 2), slice(2, a.shape[1] - 3), slice(2, a.shape[2] - 3)]
    lo = a[tuple(sl)]
    sh = list(sl)
    sh[axis] = slice(sl[axis].start + 1, sl[axis].stop + 1)
    hi = a[tuple(sh)]
    return (F32(.5) * (lo + hi)).astype(F32)


def _xxx(a):
    return a[1:a.shape[0] - 2, 2:a.shape[1] - 3, 2:a.shape[2] - 3].astype(F32)


def dump_3d(fields, base, dmpvar, cphopt=0, tubopt=0):
    """fields: dict of the level's arrays (u, v, w, pp, ptp, and qv .. ng,
    tke as the configuration has them); base: dict of 3-D base arrays ubr,
    vbr, pbr, ptbr, qvbr.  Returns (records (nvar, nz, ny, nx), names)."""
    v = (dmpvar + "x" * 16)[:16]
    out, names = [], []

    def put(name, rec):
        names.append(name)
        out.append(rec)

    if v[0] == "o":                                     # outdmp.f90:394-404
        put("ubar", _avg(base["ubr"], 2))
    if v[0] in "o-":
        put("u", _avg(fields["u"], 2))
    if v[1] == "o":                                     # :409-419
        put("vbar", _avg(base["vbr"], 1))
    if v[1] in "o-":
        put("v", _avg(fields["v"], 1))
    if v[2] == "o":                                     # :509-513
        put("w", _avg(fields["w"], 0))
    if v[3] == "o":                                     # :520-534
        put("pbar", _xxx(base["pbr"]))
        put("pp", _xxx(fields["pp"]))
    elif v[3] == "-":
        put("p", _xxx((base["pbr"] + fields["pp"]).astype(F32)))
    if v[4] == "o":                                     # :541-555
        put("ptbar", _xxx(base["ptbr"]))
        put("ptp", _xxx(fields["ptp"]))
    elif v[4] == "-":
        put("pt", _xxx((base["ptbr"] + fields["ptp"]).astype(F32)))
    if cphopt == 3:                                     # :562-635
        if v[5] == "o":
            put("qvbar", _xxx(base["qvbr"]))
        if v[5] in "o-":
            put("qv", _xxx(fields["qv"]))
        if v[6] == "o":
            for n in ("qc", "qr", "qi", "qs", "qg"):
                put(n, _xxx(fields[n]))
        if v[7] == "o":
            for n, f in (("nci", "ni"), ("ncs", "ns"), ("ncg", "ng")):
                put(n, _xxx(fields[f]))
    if tubopt >= 2 and v[11] == "o":                    # :858-862
        put("tke", _xxx(fields["tke"]))
    return (np.stack(out) if out else np.zeros((0,), F32)), names


def _record(parts):
    payload = b"".join(np.ascontiguousarray(p, F32).tobytes() for p in parts)
    n = np.uint32(len(payload)).tobytes()
    return n + payload + n


def restart_records(past, now, prec=None, phase=None, cphopt=0, tubopt=0):
    """past, now: dicts of the two levels' full arrays; prec: (5, 2, nj+2,
    ni+2) surface precipitation (rate, accumulation) of prc, prr, pri, prs,
    prg; phase: with open x, dict name -> (2, nk, nj) x phase speeds (side,
    k, j) as cress_get_phase returns them.  Returns the bytes."""
    recs = []
    one = lambda a: recs.append(_record([a]))
    for lv in (now, past):                               # outres.f90:905-935
        for n in ("u", "v", "w", "pp", "ptp"):
            one(lv[n])

    def cp(names):
        # xcpx((j,k,i), j=1..nj, k=1..nk, i=1..2) then xcpy, zero (periodic y)
        recs.append(_record([phase[n] for n in names]))
        ni = now["u"].shape[2] - 2
        nk = now["u"].shape[0]
        recs.append(_record([np.zeros((2, nk, ni), F32) for _ in names]))

    if phase is not None:                                # :939-967
        for n in ("u", "v", "w", "pp", "ptp"):
            cp([n])
    if cphopt == 3:
        one(now["qv"])                                   # :973-981
        one(past["qv"])
        if phase is not None:
            cp(["qv"])                                   # :988-992
        recs.append(_record([now["qc"], now["qr"]]))     # :999-1015
        recs.append(_record([past["qc"], past["qr"]]))
        if phase is not None:
            cp(["qc", "qr"])                             # :1031-1035
        recs.append(_record([now["qi"], now["qs"], now["qg"]]))      # :1054-1096
        recs.append(_record([now["ni"], now["ns"], now["ng"]]))
        recs.append(_record([past["qi"], past["qs"], past["qg"]]))
        recs.append(_record([past["ni"], past["ns"], past["ng"]]))
        if phase is not None:
            cp(["qi", "qs", "qg"])                       # :1106-1126
            cp(["ni", "ns", "ng"])
        recs.append(_record([prec[0, 0], prec[1, 0]]))   # prwtr(:,:,1,n), :1136-1140
        recs.append(_record([prec[0, 1], prec[1, 1]]))
        recs.append(_record([prec[2, 0], prec[3, 0], prec[4, 0]]))   # price, :1159-1163
        recs.append(_record([prec[2, 1], prec[3, 1], prec[4, 1]]))
    if tubopt == 2:
        one(now["tke"])                                  # :1280-1288
        one(past["tke"])
    return b"".join(recs)


def split_records(data):
    """The payloads (bytes) of a stream of framed records, checking each
    record's leading and trailing lengths."""
    out, off = [], 0
    while off < len(data):
        n = int(np.frombuffer(data[off:off + 4], np.uint32)[0])
        m = int(np.frombuffer(data[off + 4 + n:off + 8 + n], np.uint32)[0])
        if m != n:
            raise ValueError(f"record at {off}: lengths {n} and {m}")
        out.append(data[off + 4:off + 4 + n])
        off += 8 + n
    return out
