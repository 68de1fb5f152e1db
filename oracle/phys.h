// Oracle: physical constants and resolved run options.
//
// TEST INFRASTRUCTURE ONLY (see arr.h).
//
// Constant values restate SrcOrig/comphy.f90:49-459 (module m_comphy);
// they are held as double literals and cast to the working precision at
// the point of use, as the reference's `real` parameters are under its
// default (4-byte) and promoted (8-byte) builds.
#pragma once

namespace oracle {

struct Phys {
  static constexpr double g = 9.8;          // comphy.f90:49
  static constexpr double cp = 1004.;       // comphy.f90:61
  static constexpr double cv = 717.;        // comphy.f90:64
  static constexpr double cw = 4.218e3;     // comphy.f90:67
  static constexpr double ci = 2.106e3;     // comphy.f90:70
  static constexpr double rd = 287.;        // comphy.f90:73
  static constexpr double rv = 461.;        // comphy.f90:76
  static constexpr double epsva = .622;     // comphy.f90:79
  static constexpr double es0 = 610.78;     // comphy.f90:85
  static constexpr double p0 = 1.e5;        // comphy.f90:91
  static constexpr double t0 = 273.16;      // comphy.f90:94
  static constexpr double lv0 = 2.50078e6;  // comphy.f90:127
  static constexpr double lf0 = 3.34e5;     // comphy.f90:130
  static constexpr double ckm = .1;         // comphy.f90:341
  static constexpr double ckmin = 1.e-6;    // comphy.f90:344
  static constexpr double csnum = 0.21;     // comphy.f90:347
  static constexpr double prnum = 0.33;     // comphy.f90:350
  static constexpr double divndc = 0.05;    // comphy.f90:459
  static constexpr double omega = 7.292e-5; // comphy.f90:52
};

// Resolved namelist values for the options the hot path implements.  The
// reference resolves these through getiname/getrname (SrcOrig/getiname.f90)
// from integer ids; the oracle (like the C-ABI) receives the values.
struct Opts {
  int ni = 0, nj = 0, nk = 0;   // array dims: ni=nx+3, nj=ny+3, nk=nz+3 (setdim.f90:196-199)
  double dx = 0, dy = 0, dz = 0;   // dxiv=1.e0/dx etc. are formed in the
                                   // working precision (chknlslv.f90:432)
  int divopt = 2;     // divergence damping (pgrad.f90:260-349)
  int buyopt = 1;     // small-step buoyancy (hevi.f90:377)
  int gwmopt = 0;     // gravity-wave mode option (buoywsi.f90:163)
  double weicoe = 0.6; // HE-VI implicit weight beta (advbspi.f90:140)
  int periodic = 1;   // wbc=ebc=sbc=nbc=-1 after chknlslv maps 1->-1 on one PE
  int bbc = 2, tbc = 2;
  int fp64_solve = 0; // solve the w tridiagonal in double (product behaviour)
  int impopt = 1;     // 1 HE-VI (s_hevi), 0 HE-VE (s_heve), smalldrv.f90:370-384
  // Open (radiation) west and east boundaries: wbc = ebc = obc in {4, 5, 7}
  // (0: periodic x).  y stays periodic.  The added/subtracted boundary
  // indices iwest = ieast = 1 then narrow the 4th-order stencils
  // (sethalo.f90:535-557); gwave is the phase speed of options 5-7.
  int obc = 0;
  double gwave = 20.;
  int advopt = 2;     // 2: 4th-order horizontal advection; 3: 4th order in z too (advuvw.f90:309, advs.f90:284)
  const void* rad = nullptr;   // the run's phase speeds (openbc.h Radiation<R>)
  int iw() const { return obc ? 1 : 0; }
  int ie() const { return obc ? 1 : 0; }
};

}  // namespace oracle
