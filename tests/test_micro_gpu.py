"""GPU parity of the cold-rain microphysics (s_cloudphy, cphopt=3) and the
saturation adjustment (s_satadjst) against the CPU oracle.

The state spans warm rain, the mixed-phase layer and cold ice, sub- and
super-saturated air, so every process branch is exercised.  Tolerance:
the GPU uses the CUDA math library (expf/logf/sqrtf, <= 2 ulp) and FMA
contraction, the oracle glibc and no contraction; the microphysics has
thresholds and limiters, so a handful of cells near a branch point may
take the other branch.  We require, per field,
  * 99.9% of cells within 1e-4 * max|field| of the oracle, and
  * all cells within 5e-2 * max|field|,
and the surface precipitation (rate and accumulation) within 1e-3
relative of its maximum.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MICRO = ["ptp", "qv", "qc", "qr", "qi", "qs", "qg", "ni", "ns", "ng"]


def compare(name, g, r, tight=1e-4, loose=5e-2, frac=0.999):
    scale = float(np.abs(r).max()) + 1e-30
    err = np.abs(g - r)
    assert np.isfinite(g).all(), name
    ok = float((err <= tight * scale).mean())
    assert ok >= frac, f"{name}: only {ok:.5f} of cells within {tight} (max err {err.max():.3e}, scale {scale:.3e})"
    assert float(err.max()) <= loose * scale, f"{name}: max err {err.max():.3e} scale {scale:.3e}"


def setup_solver(cress, dims, base, dz):
    ni, nj, nk = dims
    s = cress.Solver(ni, nj, nk, 1000.0, 1000.0, dz, sthopt=1, cphopt=3)
    s.set_base3d(base)
    s.set_base_moist(base["pbr"], base["qvbr"])
    return s


@pytest.mark.parametrize("seed", [1, 2])
def test_cloudphy_matches_oracle(cress, oracle_lib, seed):
    from cress_b200 import cases
    dz = 300.0
    dims, base, past, fut, _ = cases.micro_case(37, 29, 40, dz, seed=seed)
    ni, nj, nk = dims
    ref = {k: v.copy() for k, v in fut.items()}
    prec_ref = np.zeros((5, 2, nj + 2, ni + 2), np.float32)
    npstp = oracle_lib.cloudphy(dims, base, past, ref, prec_ref, 5.0, dz)

    s = setup_solver(cress, dims, base, dz)
    for k in MICRO:
        s.put_field(k, cress.PAST, past[k])
        s.put_field(k, cress.FUTURE, fut[k])
    s.put_field("pp", cress.PAST, past["pp"])
    s.cloudphy(5.0)
    got = {k: s.get_field(k, cress.FUTURE) for k in MICRO}
    prec = s.get_precip()
    s.close()
    sl = (slice(0, nk - 1), slice(2, nj - 1), slice(2, ni - 1))   # k=1..nk-1, interior columns
    for k in MICRO:
        compare(k, got[k][sl], ref[k][sl])
    psl = (slice(None), slice(None), slice(2, nj - 1), slice(2, ni - 1))
    pscale = float(np.abs(prec_ref[psl]).max()) + 1e-30
    assert float(np.abs(prec[psl] - prec_ref[psl]).max()) <= 1e-3 * pscale
    assert npstp >= 1


def test_satadjst_matches_oracle(cress, oracle_lib):
    from cress_b200 import cases
    dz = 300.0
    dims, base, past, fut, _ = cases.micro_case(33, 27, 36, dz, seed=5)
    ni, nj, nk = dims
    st = {k: past[k].copy() for k in ("ptp", "qv", "qc", "qi", "ni")}
    oracle_lib.satadjst(dims, base["ptbr"], base["pbr"], past["pp"], st)
    s = setup_solver(cress, dims, base, dz)
    for k in ("ptp", "qv", "qc", "qi", "ni", "pp"):
        s.put_field(k, cress.NOW, past[k])
    s.satadjst(cress.NOW)
    sl = (slice(0, nk - 1), slice(2, nj - 1), slice(2, ni - 1))
    for k in ("ptp", "qv", "qc", "qi", "ni"):
        compare(k, s.get_field(k, cress.NOW)[sl], st[k][sl])
    s.close()
