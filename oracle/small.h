// Oracle: the HE-VI (impopt=1) and HE-VE (impopt=0) acoustic small steps, flat terrain
// (trnopt=0), no map factor (mfcopt=0), periodic lateral boundaries on one
// process, rigid lid / rigid bottom (bbc=tbc=2).
//
// TEST INFRASTRUCTURE ONLY (see arr.h).  This is a CPU restatement of the
// reference, used only as the parity checker; loop ranges and the
// parenthesisation of every expression follow the cited Fortran lines.
#pragma once
#include <cmath>
#include "arr.h"
#include "phys.h"
#include "openbc.h"

// OpenMP over the outermost k (or j) loop when built for the CPU baseline;
// iterations are independent, so results do not depend on the thread count.
#ifdef ORACLE_OMP
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

namespace oracle {

// Base-state and metric fields the small step reads (all `intent(in)` in
// SrcOrig/hevi.f90:106-160).
template <class R>
struct Base {
  F3<R> jcb, jcb8u, jcb8v, jcb8w;
  F3<R> rbr, ptbr, pbr, ubr, vbr, qvbr;
  F3<R> rst, rst8u, rst8v, rst8w, rcsq;
  void resize(int ni, int nj, int nk) {
    for (F3<R>* a : {&jcb, &jcb8u, &jcb8v, &jcb8w, &rbr, &ptbr, &pbr, &ubr, &vbr, &qvbr,
                     &rst, &rst8u, &rst8v, &rst8w, &rcsq})
      a->resize(ni, nj, nk);
  }
};

// s_bcycle, SrcOrig/bcycle.f90:159-225.  Periodic wrap inside one process:
// x first over j=0..nj+1 (only when wbc = ebc = -1), then y over
// i=0..ni+1 (so corners follow x).
template <class R>
void bcycle(const Opts& o, int iwsnd, int iwrcv, int iesnd, int iercv, int jssnd, int jsrcv,
            int jnsnd, int jnrcv, int kmax, F3<R>& v) {
  if (!o.periodic) return;
  const int ni = o.ni, nj = o.nj;
  if (!o.obc) {
    OMP_FOR for (int k = 1; k <= kmax; ++k)
      for (int j = 0; j <= nj + 1; ++j) v(iwrcv, j, k) = v(iesnd, j, k);
    OMP_FOR for (int k = 1; k <= kmax; ++k)
      for (int j = 0; j <= nj + 1; ++j) v(iercv, j, k) = v(iwsnd, j, k);
  }
  OMP_FOR for (int k = 1; k <= kmax; ++k)
    for (int i = 0; i <= ni + 1; ++i) v(i, jsrcv, k) = v(i, jnsnd, k);
  OMP_FOR for (int k = 1; k <= kmax; ++k)
    for (int i = 0; i <= ni + 1; ++i) v(i, jnrcv, k) = v(i, jssnd, k);
}

// s_vbcu / s_vbcv, SrcOrig/vbcu.f90:118-136 (vbcv mirrors it in y).
template <class R>
void vbcu(const Opts& o, F3<R>& uf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int j = 1; j <= nj - 1; ++j)
    for (int i = 1; i <= ni; ++i) uf(i, j, 1) = uf(i, j, 2);
  for (int j = 1; j <= nj - 1; ++j)
    for (int i = 1; i <= ni; ++i) uf(i, j, nk - 1) = uf(i, j, nk - 2);
}
template <class R>
void vbcv(const Opts& o, F3<R>& vf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni - 1; ++i) vf(i, j, 1) = vf(i, j, 2);
  for (int j = 1; j <= nj; ++j)
    for (int i = 1; i <= ni - 1; ++i) vf(i, j, nk - 1) = vf(i, j, nk - 2);
}

// s_vbcp, SrcOrig/vbcp.f90:126-160.
template <class R>
void vbcp(const Opts& o, F3<R>& ppf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  if (o.bbc == 2) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) ppf(i, j, 1) = R(2) * ppf(i, j, 2) - ppf(i, j, 3);
  } else if (o.bbc == 3) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) ppf(i, j, 1) = ppf(i, j, 2);
  }
  for (int j = 1; j <= nj - 1; ++j)
    for (int i = 1; i <= ni - 1; ++i) ppf(i, j, nk - 1) = ppf(i, j, nk - 2);
}

// s_vbcw, SrcOrig/vbcw.f90:201-499, flat terrain (j31=j32=0 so the
// terrain-following sums are zero).
template <class R>
void vbcw(const Opts& o, const Base<R>& b, const F3<R>& wc, F3<R>& wf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  if (o.bbc == 2) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) wf(i, j, 1) = -b.jcb8w(i, j, 3) * wc(i, j, 3) - R(0);
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) wf(i, j, 2) = R(0);
  } else if (o.bbc == 3) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) wf(i, j, 1) = wf(i, j, 2);
  }
  if (o.tbc == 2) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i)
        wf(i, j, nk) = -b.jcb8w(i, j, nk - 2) * wc(i, j, nk - 2) - R(0);
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) wf(i, j, nk - 1) = R(0);
  } else if (o.tbc == 3) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) wf(i, j, nk) = wf(i, j, nk - 1);
  }
}

// s_phy2cnt, SrcOrig/phy2cnt.f90:193-227 (flat terrain).
template <class R>
void phy2cnt(const Opts& o, int sthopt, const Base<R>& b, const F3<R>& w, F3<R>& wc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i)
        wc(i, j, k) = (sthopt == 0) ? w(i, j, k) : w(i, j, k) / b.jcb8w(i, j, k);
}

// s_diver3d, SrcOrig/diver3d.f90:182-326 (mfcopt=0).
template <class R>
void diver3d(const Opts& o, const F3<R>& var8u, const F3<R>& var8v, const F3<R>& var8w,
             const F3<R>& u, const F3<R>& v, const F3<R>& wc, F3<R>& div3d, F3<R>& t1, F3<R>& t2,
             F3<R>& t3) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  OMP_FOR for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni; ++i) t1(i, j, k) = var8u(i, j, k) * u(i, j, k);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni - 1; ++i) t2(i, j, k) = var8v(i, j, k) * v(i, j, k);
  }
  OMP_FOR for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) t3(i, j, k) = var8w(i, j, k) * wc(i, j, k);
  OMP_FOR for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i)
        div3d(i, j, k) = (t3(i, j, k) - t3(i, j, k + 1)) * dziv +
                         ((t1(i, j, k) - t1(i + 1, j, k)) * dxiv + (t2(i, j, k) - t2(i, j + 1, k)) * dyiv);
}

// s_diver2d, SrcOrig/diver2d.f90:166-295 (mfcopt=0).
template <class R>
void diver2d(const Opts& o, const F3<R>& var8u, const F3<R>& var8v, const F3<R>& u,
             const F3<R>& v, F3<R>& div2d, F3<R>& t1, F3<R>& t2) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy);
  OMP_FOR for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni; ++i) t1(i, j, k) = var8u(i, j, k) * u(i, j, k);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni - 1; ++i) t2(i, j, k) = var8v(i, j, k) * v(i, j, k);
  }
  OMP_FOR for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i)
        div2d(i, j, k) = (t1(i, j, k) - t1(i + 1, j, k)) * dxiv + (t2(i, j, k) - t2(i, j + 1, k)) * dyiv;
}

// s_pgrad, SrcOrig/pgrad.f90:251-395 (trnopt=0, mfcopt=0).
template <class R>
void pgrad(const Opts& o, R dts, const Base<R>& b, const F3<R>& u, const F3<R>& v,
           const F3<R>& wc, const F3<R>& pp, F3<R>& upg, F3<R>& vpg, F3<R>& wpg, F3<R>& t1,
           F3<R>& t2, F3<R>& t3) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  const R divch = R(Phys::divndc) / dts * R(o.dx) * R(o.dy);  // pgrad.f90:253
  const R divcv = R(Phys::divndc) / dts * R(o.dz) * R(o.dz);  // pgrad.f90:254
  if (o.divopt >= 1) diver3d(o, b.rst8u, b.rst8v, b.rst8w, u, v, wc, t1, t2, t3, wpg);
  if (o.divopt == 0) {
    OMP_FOR for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) t3(i, j, k) = pp(i, j, k);
  } else {
    OMP_FOR for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) t3(i, j, k) = pp(i, j, k) + divcv * b.jcb(i, j, k) * t1(i, j, k);
  }
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) wpg(i, j, k) = (t3(i, j, k - 1) - t3(i, j, k)) * dziv;
  if (o.divopt == 2) {
    OMP_FOR for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) t3(i, j, k) = pp(i, j, k) + divch * t1(i, j, k) / b.jcb(i, j, k);
  }
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) t3(i, j, k) = b.jcb(i, j, k) * t3(i, j, k);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i) upg(i, j, k) = (t3(i - 1, j, k) - t3(i, j, k)) * dxiv;
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) vpg(i, j, k) = (t3(i, j - 1, k) - t3(i, j, k)) * dyiv;
  }
}

// s_stepuv, SrcOrig/stepuv.f90:288-424: update, periodic wrap, vertical BC.
template <class R>
void stepuv(const Opts& o, R dts, const Base<R>& b, const F3<R>& ufrc, const F3<R>& vfrc,
            const F3<R>& usml, const F3<R>& vsml, F3<R>& uf, F3<R>& vf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  rbcu(o, b, uf);   // stepuv.f90:268
  rbcv(o, b, vf);   // stepuv.f90:276
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        uf(i, j, k) = uf(i, j, k) + dts * (ufrc(i, j, k) + usml(i, j, k)) / b.rst8u(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        vf(i, j, k) = vf(i, j, k) + dts * (vfrc(i, j, k) + vsml(i, j, k)) / b.rst8v(i, j, k);
  }
  bcycle(o, 3, 1, ni - 2, ni, 2, 1, nj - 2, nj - 1, nk, uf);  // stepuv.f90:390
  bcycle(o, 2, 1, ni - 2, ni - 1, 3, 1, nj - 2, nj, nk, vf);  // stepuv.f90:393
  vbcu(o, uf);
  vbcv(o, vf);
}

// s_diverpih, SrcOrig/diverpih.f90:188-214 (trnopt=0).
template <class R>
void diverpih(const Opts& o, const Base<R>& b, const F3<R>& u, const F3<R>& v, F3<R>& pdiv,
              F3<R>& t1, F3<R>& t2) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  diver2d(o, b.jcb8u, b.jcb8v, u, v, pdiv, t1, t2);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) pdiv(i, j, k) = b.rcsq(i, j, k) * pdiv(i, j, k);
}

// s_diverpiv, SrcOrig/diverpiv.f90:118-130.
template <class R>
void diverpiv(const Opts& o, const Base<R>& b, const F3<R>& w, F3<R>& pdiv) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dziv = R(1) / R(o.dz);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        pdiv(i, j, k) = b.rcsq(i, j, k) * (w(i, j, k) - w(i, j, k + 1)) * dziv;
}

// s_advbspi, SrcOrig/advbspi.f90:140-184.
template <class R>
void advbspi(const Opts& o, bool back, const Base<R>& b, const F3<R>& w, const F3<R>& pfrc,
             const F3<R>& phdiv, const F3<R>& pvdiv, F3<R>& fp) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R weicoe = R(o.weicoe);
  const R weic1m = R(1) - weicoe;
  const R g05 = R(.5) * (R)Phys::g;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        if (back)
          fp(i, j, k) = pfrc(i, j, k) + phdiv(i, j, k) +
                        weic1m * (g05 * (w(i, j, k) + w(i, j, k + 1)) * b.rst(i, j, k) + pvdiv(i, j, k));
        else
          fp(i, j, k) = fp(i, j, k) +
                        weicoe * (g05 * (w(i, j, k) + w(i, j, k + 1)) * b.rst(i, j, k) + pvdiv(i, j, k));
      }
}

// s_pgradiv, SrcOrig/pgradiv.f90:135-170.
template <class R>
void pgradiv(const Opts& o, R dts, const Base<R>& b, const F3<R>& wfrc, const F3<R>& fp,
             F3<R>& fw, F3<R>& fpdvj) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dtdzw = dts * (R(1) / R(o.dz)) * R(o.weicoe);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) fpdvj(i, j, k) = fp(i, j, k) / b.jcb(i, j, k);
  OMP_FOR for (int k = 3; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        fw(i, j, k) = wfrc(i, j, k) + fw(i, j, k) + (fpdvj(i, j, k - 1) - fpdvj(i, j, k)) * dtdzw;
}

// s_buoywsi, SrcOrig/buoywsi.f90:153-211.
template <class R>
void buoywsi(const Opts& o, R dts, const Base<R>& b, const F3<R>& pp, const F3<R>& ptp,
             const F3<R>& fp, F3<R>& fw, F3<R>& wb8s) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dtw = dts * R(o.weicoe);
  const R g05n = R(-.5) * (R)Phys::g;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        if (o.gwmopt == 0)
          wb8s(i, j, k) = (pp(i, j, k) * b.rst(i, j, k) + fp(i, j, k) * b.rbr(i, j, k) * dtw) /
                          b.rcsq(i, j, k) * g05n;
        else
          wb8s(i, j, k) = ((pp(i, j, k) * b.rst(i, j, k) + fp(i, j, k) * b.rbr(i, j, k) * dtw) /
                               b.rcsq(i, j, k) -
                           ptp(i, j, k) * b.rst(i, j, k) / b.ptbr(i, j, k)) *
                          g05n;
      }
  OMP_FOR for (int k = 3; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) fw(i, j, k) = fw(i, j, k) + (wb8s(i, j, k - 1) + wb8s(i, j, k));
}

// s_gaussel impopt=1, SrcOrig/gaussel.f90:169-262: Thomas algorithm per
// column (forward elimination, then back substitution).  S is the
// arithmetic type; the reference uses `real` (float).  Inputs are R
// arrays; the solve runs in S and the result is rounded back to R.
template <class S, class R>
void gaussel(int istr, int iend, int jstr, int jend, int kstr, int kend, const F3<R>& rr,
             const F3<R>& ss_in, const F3<R>& tt, F3<R>& ff_io) {
  const int nk = rr.nk;
  OMP_FOR for (int j = jstr; j <= jend; ++j) {
    std::vector<S> ss(nk + 2), ff(nk + 2);
    for (int i = istr; i <= iend; ++i) {
      for (int k = kstr; k <= kend; ++k) {
        ss[k] = (S)ss_in(i, j, k);
        ff[k] = (S)ff_io(i, j, k);
      }
      if (kstr == kend) {
        ff[kstr] = ff[kstr] / ss[kstr];
      } else {
        S aa = S(1) / ss[kstr];
        ss[kstr] = (S)tt(i, j, kstr) * aa;
        ff[kstr] = ff[kstr] * aa;
      }
      if (kstr + 2 <= kend) {
        for (int k = kstr + 1; k <= kend - 1; ++k) {
          S aa = S(1) / (ss[k] - (S)rr(i, j, k) * ss[k - 1]);
          ss[k] = (S)tt(i, j, k) * aa;
          ff[k] = (ff[k] - (S)rr(i, j, k) * ff[k - 1]) * aa;
        }
      }
      if (kstr + 1 <= kend) {
        S aa = S(1) / (ss[kend] - (S)rr(i, j, kend) * ss[kend - 1]);
        ff[kend] = (ff[kend] - (S)rr(i, j, kend) * ff[kend - 1]) * aa;
      }
      if (kstr + 1 <= kend) {
        for (int k = kend - 1; k >= kstr; --k) ff[k] = ff[k] - ss[k] * ff[k + 1];
      }
      for (int k = kstr; k <= kend; ++k) ff_io(i, j, k) = (R)ff[k];
    }
  }
}

// s_stepwi, SrcOrig/stepwi.f90:308-548 (buyopt 0/1, impopt=1, flat terrain).
// wc is used as scratch inside, exactly as the reference does, and is
// recomputed by phy2cnt at the end.
template <class R>
void stepwi(const Opts& o, int sthopt, R dts, const Base<R>& b, F3<R>& fw, F3<R>& wf, F3<R>& wc,
            F3<R>& t1, F3<R>& t2, F3<R>& t3) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dziv = R(1) / R(o.dz), weicoe = R(o.weicoe);
  const R g05 = R(.5) * (R)Phys::g;
  const R sbsqzi = dts * dts * weicoe * weicoe * dziv;
  const R sbsqg5 = R(.5) * (R)Phys::g * dts * dts * weicoe * weicoe;
  rbc_point(o, RV_W, nk - 1, wf);   // stepwi.f90:296
  OMP_FOR for (int k = 3; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) wf(i, j, k) = wf(i, j, k) + dts * fw(i, j, k) / b.rst8w(i, j, k);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        t1(i, j, k) = g05 * b.rbr(i, j, k) / b.rcsq(i, j, k);
        t2(i, j, k) = dziv / b.jcb(i, j, k);
      }
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        fw(i, j, k) = t1(i, j, k) + t2(i, j, k);
        wc(i, j, k) = t1(i, j, k) - t2(i, j, k);
      }
  OMP_FOR for (int k = 3; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        if (o.buyopt == 0) {
          R a = sbsqzi / b.rst8w(i, j, k);
          R mm = a * b.rcsq(i, j, k - 1);
          R nn = a * b.rcsq(i, j, k);
          t1(i, j, k) = -mm * fw(i, j, k - 1);
          t2(i, j, k) = R(1) + (nn * fw(i, j, k) - mm * wc(i, j, k - 1));
          t3(i, j, k) = nn * wc(i, j, k);
        } else {
          R rstiv = R(1) / b.rst8w(i, j, k);
          R a = rstiv * sbsqzi;
          R bb = rstiv * sbsqg5;
          R mm = bb * b.rst(i, j, k - 1) - a * b.rcsq(i, j, k - 1);
          R nn = bb * b.rst(i, j, k) + a * b.rcsq(i, j, k);
          t1(i, j, k) = mm * fw(i, j, k - 1);
          t2(i, j, k) = R(1) + (mm * wc(i, j, k - 1) + nn * fw(i, j, k));
          t3(i, j, k) = nn * wc(i, j, k);
        }
      }
  // bbcw (stepwi.f90:426) adds a terrain term that is zero on flat ground.
  if (o.fp64_solve)
    gaussel<double>(2, ni - 2, 2, nj - 2, 3, nk - 2, t1, t2, t3, wf);
  else
    gaussel<R>(2, ni - 2, 2, nj - 2, 3, nk - 2, t1, t2, t3, wf);
  bcycle(o, 2, 1, ni - 2, ni - 1, 2, 1, nj - 2, nj - 1, nk, wf);  // stepwi.f90:517
  phy2cnt(o, sthopt, b, wf, wc);                                   // stepwi.f90:540
  vbcw(o, b, wc, wf);                                              // stepwi.f90:548
}

// s_steppi, SrcOrig/steppi.f90:211-316.
template <class R>
void steppi(const Opts& o, R dts, const Base<R>& b, const F3<R>& fp, F3<R>& ppf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  rbc_point(o, RV_P, nk - 2, ppf);   // steppi.f90:199
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) ppf(i, j, k) = ppf(i, j, k) + dts * fp(i, j, k) / b.jcb(i, j, k);
  bcycle(o, 2, 1, ni - 2, ni - 1, 2, 1, nj - 2, nj - 1, nk, ppf);
  vbcp(o, ppf);
}

// Scratch owned by the caller, like the reference's tmp1..tmp6.
template <class R>
struct SmallScratch {
  F3<R> t[6];
  F3<R> x1, x2, x3;  // scratch the reference passes further down
  void resize(int ni, int nj, int nk) {
    for (auto& a : t) a.resize(ni, nj, nk);
    x1.resize(ni, nj, nk); x2.resize(ni, nj, nk); x3.resize(ni, nj, nk);
  }
};

// s_hevi, SrcOrig/hevi.f90:339-426, gwmopt=0 path (theta' is not stepped in
// the small step).
template <class R>
void hevi(const Opts& o, int sthopt, R dts, const Base<R>& b, const F3<R>& ufrc,
          const F3<R>& vfrc, const F3<R>& wfrc, const F3<R>& pfrc, const F3<R>& ptpf,
          F3<R>& uf, F3<R>& vf, F3<R>& wf, F3<R>& wc, F3<R>& ppf, SmallScratch<R>& s) {
  F3<R>&tmp1 = s.t[0], &tmp2 = s.t[1], &tmp3 = s.t[2], &tmp4 = s.t[3], &tmp5 = s.t[4], &tmp6 = s.t[5];
  // pgrad(..., uf,vf,wc,ppf, tmp1,tmp2,tmp3, tmp4,tmp5,tmp6)  hevi.f90:339
  pgrad(o, dts, b, uf, vf, wc, ppf, tmp1, tmp2, tmp3, tmp4, tmp5, tmp6);
  // stepuv(..., tmp1, tmp2 ...)                                hevi.f90:348
  stepuv(o, dts, b, ufrc, vfrc, tmp1, tmp2, uf, vf);
  // diverpih(..., uf,vf, tmp2, tmp4,tmp5,tmp6)                 hevi.f90:357
  diverpih(o, b, uf, vf, tmp2, tmp5, tmp6);
  // diverpiv(rcsq, wf, tmp4); advbspi('back', ..., tmp2,tmp4,tmp1)  hevi.f90:361-363
  diverpiv(o, b, wf, tmp4);
  advbspi(o, true, b, wf, pfrc, tmp2, tmp4, tmp1);
  // pgradiv(..., wfrc, tmp1, tmp3, tmp4)                       hevi.f90:369
  pgradiv(o, dts, b, wfrc, tmp1, tmp3, tmp4);
  // buoywsi(..., ppf, ptpf, tmp1, tmp3, tmp4)                  hevi.f90:377
  if (o.buyopt == 1) buoywsi(o, dts, b, ppf, ptpf, tmp1, tmp3, tmp4);
  // stepwi(..., tmp3, wf, wc, tmp4,tmp5,tmp6)                  hevi.f90:408
  stepwi(o, sthopt, dts, b, tmp3, wf, wc, tmp4, tmp5, tmp6);
  // diverpiv; advbspi('fore', ..., tmp3,tmp4,tmp1)             hevi.f90:418-420
  diverpiv(o, b, wf, tmp4);
  advbspi(o, false, b, wf, pfrc, tmp3, tmp4, tmp1);
  // steppi(..., tmp1, ppf)                                     hevi.f90:426
  steppi(o, dts, b, tmp1, ppf);
}

// s_buoywse, SrcOrig/buoywse.f90:135-187 (gwmopt=0, lines 151 and 184): the explicit small-step
// buoyancy added to wsml (which holds the vertical pressure gradient).
template <class R>
void buoywse(const Opts& o, const Base<R>& b, const F3<R>& pp, F3<R>& wsml, F3<R>& wb8s) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R g05n = R(-.5) * (R)Phys::g;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) wb8s(i, j, k) = pp(i, j, k) * b.rst(i, j, k) / b.rcsq(i, j, k) * g05n;
  OMP_FOR for (int k = 3; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) wsml(i, j, k) = wsml(i, j, k) + (wb8s(i, j, k - 1) + wb8s(i, j, k));
}

// s_stepwe, SrcOrig/stepwe.f90:255-370 (update at 261): explicit w update, periodic wrap,
// contravariant w and the vertical boundary rows.
template <class R>
void stepwe(const Opts& o, int sthopt, R dts, const Base<R>& b, const F3<R>& wfrc, const F3<R>& wsml,
            F3<R>& wf, F3<R>& wc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        wf(i, j, k) = wf(i, j, k) + dts * (wfrc(i, j, k) + wsml(i, j, k)) / b.rst8w(i, j, k);
  bcycle(o, 2, 1, ni - 2, ni - 1, 2, 1, nj - 2, nj - 1, nk, wf);  // stepwe.f90:337
  phy2cnt(o, sthopt, b, wf, wc);                                   // stepwe.f90:360
  vbcw(o, b, wc, wf);                                              // stepwe.f90:368
}

// s_diverpe, SrcOrig/diverpe.f90:153-169: rcsq times the 3-D divergence of
// the J-weighted new winds.
template <class R>
void diverpe(const Opts& o, const Base<R>& b, const F3<R>& u, const F3<R>& v, const F3<R>& wc, F3<R>& pdiv,
             F3<R>& t1, F3<R>& t2, F3<R>& t3) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  diver3d(o, b.jcb8u, b.jcb8v, b.jcb8w, u, v, wc, pdiv, t1, t2, t3);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) pdiv(i, j, k) = b.rcsq(i, j, k) * pdiv(i, j, k);
}

// s_advbspe, SrcOrig/advbspe.f90:118-135 (127).
template <class R>
void advbspe(const Opts& o, const Base<R>& b, const F3<R>& w, const F3<R>& pdiv, F3<R>& psml) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R g05 = R(.5) * (R)Phys::g;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        psml(i, j, k) = g05 * (w(i, j, k) + w(i, j, k + 1)) * b.rst(i, j, k) + pdiv(i, j, k);
}

// s_steppe, SrcOrig/steppe.f90:218-323 (update at 224).
template <class R>
void steppe(const Opts& o, R dts, const Base<R>& b, const F3<R>& pfrc, const F3<R>& psml, F3<R>& ppf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        ppf(i, j, k) = ppf(i, j, k) + dts * (pfrc(i, j, k) + psml(i, j, k)) / b.jcb(i, j, k);
  bcycle(o, 2, 1, ni - 2, ni - 1, 2, 1, nj - 2, nj - 1, nk, ppf);
  vbcp(o, ppf);
}

// s_heve, SrcOrig/heve.f90:337-406, gwmopt=0 path.
template <class R>
void heve(const Opts& o, int sthopt, R dts, const Base<R>& b, const F3<R>& ufrc, const F3<R>& vfrc,
          const F3<R>& wfrc, const F3<R>& pfrc, F3<R>& uf, F3<R>& vf, F3<R>& wf, F3<R>& wc, F3<R>& ppf,
          SmallScratch<R>& s) {
  F3<R>&tmp1 = s.t[0], &tmp2 = s.t[1], &tmp3 = s.t[2], &tmp4 = s.t[3], &tmp5 = s.t[4], &tmp6 = s.t[5];
  pgrad(o, dts, b, uf, vf, wc, ppf, tmp1, tmp2, tmp3, tmp4, tmp5, tmp6);   // heve.f90:337
  stepuv(o, dts, b, ufrc, vfrc, tmp1, tmp2, uf, vf);                       // heve.f90:346
  if (o.buyopt == 1) buoywse(o, b, ppf, tmp3, tmp4);                        // heve.f90:356
  stepwe(o, sthopt, dts, b, wfrc, tmp3, wf, wc);                            // heve.f90:386
  diverpe(o, b, uf, vf, wc, tmp2, tmp3, tmp4, tmp5);                        // heve.f90:395
  advbspe(o, b, wf, tmp2, tmp1);                                            // heve.f90:398
  steppe(o, dts, b, pfrc, tmp1, ppf);                                       // heve.f90:404
}

// One substep of s_smalldrv's loop: s_heve for impopt=0, s_hevi otherwise
// (smalldrv.f90:370-398).
template <class R>
void small_substep(const Opts& o, int sthopt, R dts, const Base<R>& b, const F3<R>& ufrc, const F3<R>& vfrc,
                   const F3<R>& wfrc, const F3<R>& pfrc, const F3<R>& ptpf, F3<R>& uf, F3<R>& vf, F3<R>& wf,
                   F3<R>& wc, F3<R>& ppf, SmallScratch<R>& s) {
  if (o.impopt == 0) heve<R>(o, sthopt, dts, b, ufrc, vfrc, wfrc, pfrc, uf, vf, wf, wc, ppf, s);
  else hevi<R>(o, sthopt, dts, b, ufrc, vfrc, wfrc, pfrc, ptpf, uf, vf, wf, wc, ppf, s);
}

}  // namespace oracle
