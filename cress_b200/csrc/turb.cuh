// Smagorinsky turbulence: deformation-tensor components on the fly
// (internal).  Every component is formed from the past winds where a
// kernel needs it, in the reference's operation order, instead of being
// stored as the reference's t11..t32 arrays (SrcOrig/defomten.f90:305-1091,
// trnopt=0, mfcopt=0, periodic, flat terrain).
//
// The winds and the 1-D columns come through accessors, so one set of
// formulas serves kernels that read global memory and kernels that read a
// shared-memory tile: U(x, y, z), V(.), W(.) give the past u, v, w at the
// offset (x, y, z) from the kernel's point of level k, C(field, kk) a
// column value of level kk (base or derived, forcing.cuh).  The values are
// float, or F2 (f2.cuh) for a pair of points.
#pragma once
#include "forcing.cuh"
#include "hevi.cuh"

namespace cress {

template <class FC, class FU, class FV, class FW>
struct DeformAt {
  const FC& C;
  const FU& U;
  const FV& V;
  const FW& W;
  int k, nk;
  float dxiv, dyiv, dziv;

  // s11, s22, s33 at the scalar point (x, y, z) (defomten.f90:471-500, 667-686)
  __device__ __forceinline__ auto s11(int x, int y, int z) const {
    const int kk = k + z;
    const float j8u = C(C_JCB8U, kk);
    const auto d = (U(x + 1, y, z) * j8u - U(x, y, z) * j8u) * dxiv;
    return C(D_2JCB, kk) * d;
  }
  __device__ __forceinline__ auto s22(int x, int y, int z) const {
    const int kk = k + z;
    const float j8v = C(C_JCB8V, kk);
    const auto d = (V(x, y + 1, z) * j8v - V(x, y, z) * j8v) * dyiv;
    return C(D_2JCB, kk) * d;
  }
  __device__ __forceinline__ auto s33(int x, int y, int z) const {
    return C(D_2JCB, k + z) * (W(x, y, z + 1) - W(x, y, z)) * dziv;
  }
  // s12 at the u-v corner (x, y, z) (defomten.f90:336-352, 471-480)
  __device__ __forceinline__ auto s12(int x, int y, int z) const {
    const int kk = k + z;
    const float j8u = C(C_JCB8U, kk), j8v = C(C_JCB8V, kk);
    const float t3 = C(D_4JCB, kk);
    return t3 * ((U(x, y, z) * j8u - U(x, y - 1, z) * j8u) * dyiv + (V(x, y, z) * j8v - V(x - 1, y, z) * j8v) * dxiv);
  }
  // s13 = s31 at the u-w point (x, y, z), level 2..nk-1 (defomten.f90:763-833)
  __device__ __forceinline__ auto s13(int x, int y, int z) const {
    const float j8w = C(C_JCB8W, k + z);
    const float t3 = C(D_2J8W, k + z);
    return ((W(x, y, z) * j8w - W(x - 1, y, z) * j8w) * dxiv + (U(x, y, z) - U(x, y, z - 1)) * dziv) * t3;
  }
  // s23 = s32 at the v-w point (x, y, z), level 2..nk-1 (defomten.f90:934-986)
  __device__ __forceinline__ auto s23(int x, int y, int z) const {
    const float j8w = C(C_JCB8W, k + z);
    const float t3 = C(D_2J8W, k + z);
    return ((W(x, y, z) * j8w - W(x, y - 1, z) * j8w) * dyiv + (V(x, y, z) - V(x, y, z - 1)) * dziv) * t3;
  }
  // s31, s32 with the rigid-lid images of s_bcten at levels 1 and nk
  // (bcten.f90:126-160: ten(1) = -ten(3), ten(nk) = -ten(nk-2))
  __device__ __forceinline__ auto s31(int x, int y, int z) const {
    const int kk = k + z;
    if (kk == 1) return -s13(x, y, z + 2);
    if (kk == nk) return -s13(x, y, z - 2);
    return s13(x, y, z);
  }
  __device__ __forceinline__ auto s32(int x, int y, int z) const {
    const int kk = k + z;
    if (kk == 1) return -s23(x, y, z + 2);
    if (kk == nk) return -s23(x, y, z - 2);
    return s23(x, y, z);
  }
};

template <class FC, class FU, class FV, class FW>
__device__ __forceinline__ DeformAt<FC, FU, FV, FW> deform_at(const FC& C, const FU& U, const FV& V, const FW& W,
                                                              int k, int nk, float dxiv, float dyiv, float dziv) {
  return DeformAt<FC, FU, FV, FW>{C, U, V, W, k, nk, dxiv, dyiv, dziv};
}

}  // namespace cress
