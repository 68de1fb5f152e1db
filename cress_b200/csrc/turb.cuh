// Smagorinsky turbulence: deformation-tensor components on the fly
// (internal).  Every component is formed from the past winds where a
// kernel needs it, in the reference's operation order, instead of being
// stored as the reference's t11..t32 arrays (SrcOrig/defomten.f90:305-1091,
// trnopt=0, mfcopt=0, periodic, flat terrain).
#pragma once
#include "hevi.cuh"

namespace cress {

struct Deform {
  const float* col;
  int nc, nk;
  const float *u, *v, *w;
  long long px, pl;
  float dxiv, dyiv, dziv;

  __device__ __forceinline__ float C(int f, int k) const { return __ldg(col + f * nc + k); }
  __device__ __forceinline__ float U(long long p) const { return __ldg(u + p); }
  __device__ __forceinline__ float V(long long p) const { return __ldg(v + p); }
  __device__ __forceinline__ float W(long long p) const { return __ldg(w + p); }

  // s11, s22, s33 at the scalar point p of level k (defomten.f90:471-500, 667-686)
  __device__ __forceinline__ float s11(long long p, int k) const {
    const float j8u = C(C_JCB8U, k);
    const float d = (U(p + 1) * j8u - U(p) * j8u) * dxiv;
    return (2.f / C(C_JCB, k)) * d;
  }
  __device__ __forceinline__ float s22(long long p, int k) const {
    const float j8v = C(C_JCB8V, k);
    const float d = (V(p + px) * j8v - V(p) * j8v) * dyiv;
    return (2.f / C(C_JCB, k)) * d;
  }
  __device__ __forceinline__ float s33(long long p, int k) const {
    return (2.f / C(C_JCB, k)) * (W(p + pl) - W(p)) * dziv;
  }
  // s12 at the u-v corner p = (i, j) of level k (defomten.f90:336-352, 471-480)
  __device__ __forceinline__ float s12(long long p, int k) const {
    const float jc = C(C_JCB, k), j8u = C(C_JCB8U, k), j8v = C(C_JCB8V, k);
    const float t3 = 4.f / ((jc + jc) + (jc + jc));
    return t3 * ((U(p) * j8u - U(p - px) * j8u) * dyiv + (V(p) * j8v - V(p - 1) * j8v) * dxiv);
  }
  // s13 = s31 at the u-w point p of level kk = 2..nk-1 (defomten.f90:763-833)
  __device__ __forceinline__ float s13(long long p, int kk) const {
    const float j8w = C(C_JCB8W, kk);
    const float t3 = 2.f / (j8w + j8w);
    return ((W(p) * j8w - W(p - 1) * j8w) * dxiv + (U(p) - U(p - pl)) * dziv) * t3;
  }
  // s23 = s32 at the v-w point p of level kk = 2..nk-1 (defomten.f90:934-986)
  __device__ __forceinline__ float s23(long long p, int kk) const {
    const float j8w = C(C_JCB8W, kk);
    const float t3 = 2.f / (j8w + j8w);
    return ((W(p) * j8w - W(p - px) * j8w) * dyiv + (V(p) - V(p - pl)) * dziv) * t3;
  }
  // s31, s32 with the rigid-lid images of s_bcten at kk = 1 and nk
  // (bcten.f90:126-160: ten(1) = -ten(3), ten(nk) = -ten(nk-2))
  __device__ __forceinline__ float s31(long long p, int kk) const {
    if (kk == 1) return -s13(p + 2 * pl, 3);
    if (kk == nk) return -s13(p - 2 * pl, nk - 2);
    return s13(p, kk);
  }
  __device__ __forceinline__ float s32(long long p, int kk) const {
    if (kk == 1) return -s23(p + 2 * pl, 3);
    if (kk == nk) return -s23(p - 2 * pl, nk - 2);
    return s23(p, kk);
  }
};

}  // namespace cress
