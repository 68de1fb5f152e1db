// Cold-rain bulk microphysics (s_cloudphy -> s_coldblk, cphopt=3,
// haiopt=0) and saturation adjustment (s_satadjst) for sm_100a.
//
// k_micro_src (one thread per cell, interior columns, k = 1..nk-1, the
// reference's range): getvdens/getexner/diagnw, adjstni on the future
// level, termblk on the past level, every process rate of srcblk held in
// registers (the reference keeps 77 scratch 3-D arrays, SrcOrig/comblk.f90),
// adjstni again; it writes the ten future fields and folds each cell's
// sedimentation CFL limit dz*jcb/(u+eps) into one domain minimum
// (the chkfall allreduce of SrcOrig/fallblk.f90:439) with a warp reduction
// and one atomicMin per warp.
// k_micro_fall (one thread per column and sedimenting species; the eight
// species are independent): recovers npstp and dtp from that minimum
// (fallblk.f90:441-449) and runs the upwind sedimentation sub-steps of its
// species column (upwqp.f90:160-225, upwnp.f90:140-176) with the past-level
// fall speeds k_micro_src stored, and the surface precipitation rate and
// accumulation; k_adjstni then applies the final adjstni (coldblk.f90:469).
#include <cuda_runtime.h>
#include "common.cuh"
#include "hevi.cuh"
#include "micro.cuh"
#include "coldrain.cuh"
#include "mlp.cuh"
#include "mlp_impl.cuh"

namespace cress {

namespace {


__device__ inline void load_cell(const MicroArgs& a, long long id, int k, MCell& c) {
  const int nc = a.g.nk + 1;
  const float rddvcp = 287.f / 1004.f, p0iv = 1.f / 1.e5f;
  c.ptbr = __ldg(a.col + C_PTBR * nc + k);
  c.rbr = __ldg(a.col + C_RBR * nc + k);
  c.rbv = 1.f / c.rbr;                                                  // getvdens.f90:106
  c.p = __ldg(a.col + C_PBR * nc + k) + __ldg(a.ppp + id);              // getexner.f90:129
  c.pi = expf(rddvcp * logf(p0iv * c.p));                               // getexner.f90:131
  c.ptpp = __ldg(a.ptpp + id); c.qvp = __ldg(a.qvp + id); c.qcp = __ldg(a.qcp + id);
  c.qrp = __ldg(a.qrp + id); c.qip = __ldg(a.qip + id); c.qsp = __ldg(a.qsp + id);
  c.qgp = __ldg(a.qgp + id); c.ncip = __ldg(a.nip + id); c.ncsp = __ldg(a.nsp + id);
  c.ncgp = __ldg(a.ngp + id);
  diagnw_cell(c.rbr, c.qrp, c.nccp, c.ncrp);                           // cloudphy.f90:366
}

// The fall speeds of the past level (termblk) in the order the
// sedimentation kernel runs the species: cloud water, cloud ice, ice
// number, rain, snow, graupel, snow number, graupel number.
__device__ __forceinline__ void store_speeds(const MicroArgs& a, long long id, const MCell& c) {
  const long long n3 = (long long)a.g.plane * a.g.nk;
  float* u = a.uspd + id;
  u[0] = c.ucq; u[n3] = c.uiq; u[2 * n3] = c.uin; u[3 * n3] = c.urq;
  u[4 * n3] = c.usq; u[5 * n3] = c.ugq; u[6 * n3] = c.usn; u[7 * n3] = c.ugn;
}

__global__ void __launch_bounds__(256, 3) k_micro_src(const MicroArgs a) {
  const Grid g = a.g;
  const int i = col_lo(g) + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  const bool in = i <= col_hi(g) && j <= g.nj - 2 && k <= g.nk - 1;
  float lim = 3.0e38f;
  if (in) {
    const long long id = g.at(i, j, k);
    MCell c;
    load_cell(a, id, k, c);
    c.ptpf = a.ptpf[id]; c.qvf = a.qvf[id]; c.qcf = a.qcf[id]; c.qrf = a.qrf[id];
    c.qif = a.qif[id]; c.qsf = a.qsf[id]; c.qgf = a.qgf[id]; c.ncif = a.nif[id];
    c.ncsf = a.nsf[id]; c.ncgf = a.ngf[id];
    adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);   // coldblk.f90:327
    termblk_cell(a.thresq, c);                                                // coldblk.f90:344
    store_speeds(a, id, c);
    srcblk_cell(a.dtb, a.thresq, c);                                          // coldblk.f90:356
    adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);   // coldblk.f90:425
    a.ptpf[id] = c.ptpf; a.qvf[id] = c.qvf; a.qcf[id] = c.qcf; a.qrf[id] = c.qrf;
    a.qif[id] = c.qif; a.qsf[id] = c.qsf; a.qgf[id] = c.qgf; a.nif[id] = c.ncif;
    a.nsf[id] = c.ncsf; a.ngf[id] = c.ncgf;
    // fallblk.f90:362-377 (flqcqi_opt=1: cloud water and ice fall too)
    const float eps = 1.e-20f;
    const float dzjcb = a.dz * __ldg(a.col + C_JCB * (g.nk + 1) + k);
    lim = fminf(lim, dzjcb / (c.ucq + eps));
    lim = fminf(lim, dzjcb / (c.urq + eps));
    lim = fminf(lim, dzjcb / (c.uiq + eps));
    lim = fminf(lim, dzjcb / (c.usq + eps));
    lim = fminf(lim, dzjcb / (c.ugq + eps));
  }
  for (int o = 16; o > 0; o >>= 1) lim = fminf(lim, __shfl_xor_sync(0xffffffffu, lim, o));
  if ((threadIdx.x & 31) == 0 && lim < 3.0e38f) atomicMin(a.dtp_bits, __float_as_int(lim));
}

// One thread per column and species (blockIdx.z).  npstp upwind sub-steps
// of s_upwqp / s_upwnp (upwqp.f90:160-225, upwnp.f90:140-176) stream up the
// column: the flux rbr*u*q of level k+1 is formed from the not yet updated
// q(k+1) while q(k) is written, so a sub-step is one read and one write of
// the column; the surface rate (flx(1)+flx(2))/2/rhow accumulates over
// the sub-steps.
__global__ void __launch_bounds__(128) k_micro_fall(const MicroArgs a) {
  const Grid g = a.g;
  const int nk = g.nk;
  const int i = col_lo(g) + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int f = blockIdx.z;
  if (i > col_hi(g) || j > g.nj - 2) return;
  // fallblk.f90:421-449
  const float dtb = a.dtb;
  float dtp = fminf(__int_as_float(*a.dtp_bits), dtb);
  int npstp;
  if (dtp < dtb) {
    npstp = (int)((dtb + .001f) / dtp) + 1;
    dtp = dtb / (float)npstp;
  } else {
    npstp = 1;
    dtp = dtb;
  }
  const float dziv = 1.f / a.dz;
  const float dzvdt = dziv * dtp;
  const float rwiv05 = .5f / 1.e3f, dtp05 = .5f * dtp;
  const int nc = nk + 1;
  const float* crbr = a.col + C_RBR * nc;
  const float* crst = a.col + C_RST * nc;
  const long long id1 = g.at(i, j, 1);
  const long long pl = g.plane;
  const long long n3 = pl * nk;
  const long long pp2 = (long long)g.px * g.py;
  const long long pid = (long long)j * g.px + i;
  // species f: qc, qi, ni, qr, qs, qg, ns, ng; its precipitation slot
  // (prc, pri, -, prr, prs, prg, -, -)
  float* const field = f == 0 ? a.qcf : f == 1 ? a.qif : f == 2 ? a.nif : f == 3 ? a.qrf
                     : f == 4 ? a.qsf : f == 5 ? a.qgf : f == 6 ? a.nsf : a.ngf;
  const int s = f == 0 ? 0 : f == 1 ? 2 : f == 3 ? 1 : f == 4 ? 3 : f == 5 ? 4 : -1;
  {
    float* fld = field + id1;
    const float* u = a.uspd + f * n3 + id1;
    float rate = 0.f, acc = 0.f;
    if (s >= 0) { rate = a.prec[(2 * s) * pp2 + pid]; acc = a.prec[(2 * s + 1) * pp2 + pid]; }
#pragma unroll 1
    for (int it = 0; it < npstp; ++it) {
      float q0 = fld[0];
      float f0 = __ldg(crbr + 1) * __ldg(u) * q0;
      const float flx1 = f0;
      float flx2 = 0.f, qn = 0.f;
#pragma unroll 4
      for (int k = 1; k <= nk - 2; ++k) {
        const long long o = (long long)k * pl;             // level k+1
        const float q1 = fld[o];
        const float f1 = __ldg(crbr + k + 1) * __ldg(u + o) * q1;
        if (k == 1) flx2 = f1;
        qn = fmaxf(q0 + (f1 - f0) / __ldg(crst + k) * dzvdt, 0.f);
        fld[o - pl] = qn;
        q0 = q1;
        f0 = f1;
      }
      fld[(long long)(nk - 2) * pl] = qn;                   // q(nk-1) = q(nk-2)
      if (s >= 0) {
        rate = (flx1 + flx2) * rwiv05;
        acc = acc + rate * dtp05;
      }
    }
    if (s >= 0) { a.prec[(2 * s) * pp2 + pid] = rate; a.prec[(2 * s + 1) * pp2 + pid] = acc; }
  }
}

// coldblk.f90:467-470: adjstni once more after the sedimentation
// (flqcqi_opt=1), interior points, k = 1..nk-1.
__global__ void __launch_bounds__(256) k_adjstni(const MicroArgs a) {
  const Grid g = a.g;
  const int i = col_lo(g) + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > col_hi(g) || j > g.nj - 2 || k > g.nk - 1) return;
  const long long id = g.at(i, j, k);
  const float rb = __ldg(a.col + C_RBR * (g.nk + 1) + k), rbv = 1.f / rb;
  float nci = a.nif[id], ncs = a.nsf[id], ncg = a.ngf[id];
  adjstni_cell(rb, rbv, a.qif[id], a.qsf[id], a.qgf[id], nci, ncs, ncg);
  a.nif[id] = nci; a.nsf[id] = ncs; a.ngf[id] = ncg;
}

__global__ void k_init_dtp(int* dtp_bits, float v) { *dtp_bits = __float_as_int(v); }

// s_satadjst (cphopt=3): siadjst then swadjst on one level.
__global__ void __launch_bounds__(256) k_satadjst(const SatArgs a) {
  const Grid g = a.g;
  const int i = col_lo(g) + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > col_hi(g) || j > g.nj - 2 || k > g.nk - 1) return;
  const long long id = g.at(i, j, k);
  const int nc = g.nk + 1;
  const float rddvcp = 287.f / 1004.f, p0iv = 1.f / 1.e5f;
  const float p = __ldg(a.col + C_PBR * nc + k) + __ldg(a.pp + id);     // getexner.f90:129
  const float pi = expf(rddvcp * logf(p0iv * p));
  float ptp = a.ptp[id], qv = a.qv[id], qc = a.qc[id], qi = a.qi[id], ni = a.ni[id];
  satadjst_cell(a.thresq, __ldg(a.col + C_PTBR * nc + k), pi, p, ptp, qv, qc, qi, ni);
  a.ptp[id] = ptp; a.qv[id] = qv; a.qc[id] = qc; a.qi[id] = qi; a.ni[id] = ni;
}

// In a large step: cloudphy's final adjstni on t+dt (coldblk.f90:469; the
// dry filter that runs in between does not touch these fields), s_timeflt
// for the moist fields (timeflt.f90:405-520), then s_satadjst on t and
// t+dt (intgdrv.f90:985-998), interior points, k = 1..nk-1.
__global__ void __launch_bounds__(256) k_moist_post(const MoistPostArgs a) {
  const Grid g = a.g;
  const int i = col_lo(g) + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > col_hi(g) || j > g.nj - 2 || k > g.nk - 1) return;
  const long long id = g.at(i, j, k);
  const int nc = g.nk + 1;
  // every load before the first store, so they are all in flight at once
  // (the stores could alias them as far as the compiler knows)
  float c[9], fv[9], pv[9];
#pragma unroll
  for (int n = 0; n < 9; ++n) {
    c[n] = a.c[n][id];
    fv[n] = a.f[n][id];
    if (a.filter) pv[n] = __ldg(a.p[n] + id);
  }
  const float ppc = a.ppc[id], ptpc = a.ptpc[id], ppf = a.ppf[id], ptpf = a.ptpf[id];
  if (a.adjstni) {   // what k_adjstni does, on the future numbers
    const float rb = __ldg(a.col + C_RBR * nc + k), rbv = 1.f / rb;
    adjstni_cell(rb, rbv, fv[3], fv[4], fv[5], fv[6], fv[7], fv[8]);
    a.f[6][id] = fv[6]; a.f[7][id] = fv[7]; a.f[8][id] = fv[8];
  }
  if (a.filter) {
    const float fc = a.filcoe, m1fc2 = 1.f - 2.f * a.filcoe;
#pragma unroll
    for (int n = 0; n < 9; ++n) {
      c[n] = m1fc2 * c[n] + fc * (fv[n] + pv[n]);
      if (n != 0 && n != 1 && n != 3 && n != 6) a.c[n][id] = c[n];
    }
  }
  const float rddvcp = 287.f / 1004.f, p0iv = 1.f / 1.e5f;
  const float pbr = __ldg(a.col + C_PBR * nc + k), ptbr = __ldg(a.col + C_PTBR * nc + k);
  {
    const float p = pbr + ppc;                                          // getexner.f90:129
    const float pi = expf(rddvcp * logf(p0iv * p));
    float ptp = ptpc;
    satadjst_cell(a.thresq, ptbr, pi, p, ptp, c[0], c[1], c[3], c[6]);
    a.ptpc[id] = ptp;
    a.c[0][id] = c[0]; a.c[1][id] = c[1]; a.c[3][id] = c[3]; a.c[6][id] = c[6];
  }
  {
    const float p = pbr + ppf;
    const float pi = expf(rddvcp * logf(p0iv * p));
    float ptp = ptpf, qv = fv[0], qc = fv[1], qi = fv[3], ni = fv[6];
    satadjst_cell(a.thresq, ptbr, pi, p, ptp, qv, qc, qi, ni);
    a.ptpf[id] = ptp;
    a.f[0][id] = qv; a.f[1][id] = qc; a.f[3][id] = qi; a.f[6][id] = ni;
  }
}

}  // namespace

int micro_init_tables() {
  // SrcOrig/setref.f90:473-601
  static const float c[41] = {0.f, .7939e-10f, .7841e-9f, .3369e-8f, .4336e-8f, .5285e-8f, .3728e-8f,
                              .1852e-8f, .2991e-9f, .4248e-9f, .7434e-9f, .1812e-8f, .4394e-8f,
                              .9145e-8f, .1725e-7f, .3348e-7f, .1725e-7f, .9175e-8f, .4412e-8f,
                              .2252e-8f, .9115e-9f, .4876e-9f, .3473e-9f, .4758e-9f, .6306e-9f,
                              .8573e-9f, .7868e-9f, .7192e-9f, .6513e-9f, .5956e-9f, .5333e-9f,
                              .4834e-9f, .4335e-9f, .3836e-9f, .3337e-9f, .2838e-9f, .2339e-9f,
                              .1840e-9f, .1341e-9f, .8420e-10f, .3430e-10f};
  static const float p[41] = {0.f, .4006f, .4831f, .5320f, .5307f, .5319f, .5249f, .4888f, .3894f,
                              .4047f, .4318f, .4771f, .5183f, .5463f, .5651f, .5813f, .5655f, .5478f,
                              .5203f, .4906f, .4447f, .4126f, .3960f, .4149f, .4320f, .4506f, .4483f,
                              .4460f, .4433f, .4413f, .4382f, .4361f, .4340f, .4319f, .4298f, .4277f,
                              .4256f, .4235f, .4214f, .4193f, .4172f};
  float ck[41];
  for (int n = 0; n <= 40; ++n) ck[n] = c[n] * expf(3.f * p[n] * 2.30259f);   // setref.f90:559-600
  if (cudaMemcpyToSymbol(kKoeC, ck, sizeof ck) != cudaSuccess) return CRESS_E_CUDA;
  if (cudaMemcpyToSymbol(kKoeP, p, sizeof p) != cudaSuccess) return CRESS_E_CUDA;
  return CRESS_OK;
}

// s_fallblk for the eight species, then the final adjstni (two launches;
// one when k_moist_post applies the adjstni).
static void launch_fall(const MicroArgs& a, cudaStream_t st) {
  dim3 b2(32, 4, 1);
  dim3 gr2((ncols(a.g) + 31) / 32, (a.g.nj - 3 + 3) / 4, 8);
  k_micro_fall<<<gr2, b2, 0, st>>>(a);
  if (a.defer_adjstni) return;
  dim3 b(32, 8, 1);
  dim3 gr((ncols(a.g) + 31) / 32, (a.g.nj - 3 + 7) / 8, a.g.nk - 1);
  k_adjstni<<<gr, b, 0, st>>>(a);
}

// The process rates and the sub-step minimum (two launches), then the
// sedimentation (two launches); a y-slab rank reduces the minimum over
// the ranks in between.
int launch_cloudphy_src(const MicroArgs& a, cudaStream_t st) {
  k_init_dtp<<<1, 1, 0, st>>>(a.dtp_bits, a.dtb);
  dim3 b(32, 8, 1);
  dim3 gr((ncols(a.g) + 31) / 32, (a.g.nj - 3 + 7) / 8, a.g.nk - 1);
  k_micro_src<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_cloudphy_fall(const MicroArgs& a, cudaStream_t st) {
  launch_fall(a, st);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_cloudphy(const MicroArgs& a, cudaStream_t st) {
  int rc = launch_cloudphy_src(a, st);
  return rc ? rc : launch_cloudphy_fall(a, st);
}

int launch_moist_post(const MoistPostArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((ncols(a.g) + 31) / 32, (a.g.nj - 3 + 7) / 8, a.g.nk - 1);
  k_moist_post<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_satadjst(const SatArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((ncols(a.g) + 31) / 32, (a.g.nj - 3 + 7) / 8, a.g.nk - 1);
  k_satadjst<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

// Learned-form kernels (they use this file's Koenig tables and loaders).
#include "micro_learned.cuh"
#include "mlp_fused.cuh"

namespace cress {

int launch_collect_tuples(const MicroArgs& a, const float* w, Mlp* m, int stride, float keep_zero,
                          unsigned long long seed, unsigned long long* count_d, cudaStream_t st) {
  if (stride < 1) return CRESS_E_ARG;
  // append after the tuples already stored
  k_micro_tuples<<<148 * 8, 128, 0, st>>>(a, w, m->tx + m->ntup * kMlpIn, m->ty + m->ntup * kMlpOut, count_d,
                                          m->tcap - m->ntup, stride, keep_zero, seed);
  return cudaGetLastError() == cudaSuccess ? CRESS_OK : CRESS_E_CUDA;
}

// s_cloudphy with the MLP in place of the process-rate part: chunks of
// `L.chunk` interior cells go through features -> 4 tensor-core GEMMs ->
// application; rejected cells run the plain process rates; then the plain
// sedimentation.
int launch_cloudphy_learned(const MicroArgs& a, const float* w, Mlp* m, const LearnedBuffers& L, float resid_tol,
                            cudaStream_t st, long long* launches) {
  k_init_dtp<<<1, 1, 0, st>>>(a.dtp_bits, a.dtb);
  ++*launches;
  const long long ncell = (long long)(a.g.ni - 3) * (a.g.nj - 3) * (a.g.nk - 1);
  for (long long n0 = 0; n0 < ncell; n0 += L.chunk) {
    const int cnt = (int)((ncell - n0) < L.chunk ? (ncell - n0) : L.chunk);
    const int rows = (cnt + 127) / 128 * 128;
    k_mlp_features<<<rows / 128, 128, 0, st>>>(a, w, n0, cnt, rows, m->norm_d, L.xb, L.env);
    int rc;
    const bf16* in = L.xb;
    int kin = kMlpK1;
    const bf16* wt[3] = {m->w.w1t, m->w.w2t, m->w.w3t};
    const int boff[3] = {MlpLayout::B1, MlpLayout::B2, MlpLayout::B3};
    bf16* outs[3] = {L.h0, L.h1, L.h0};
    for (int l = 0; l < 3; ++l) {
      GemmArgs g{};
      g.M = rows; g.N = kMlpH; g.K = kin;
      g.bias = m->params + boff[l];
      g.act = 1;
      g.out_bf = outs[l]; g.ldb = kMlpH;
      g.err = L.err;
      if ((rc = gemm_bf16(in, kin, wt[l], kin, g, st))) return rc;
      in = outs[l];
      kin = kMlpH;
    }
    GemmArgs g{};
    g.M = rows; g.N = kMlpN4; g.K = kMlpH;
    g.bias = m->params + MlpLayout::B4;
    g.out_f32 = L.y; g.ldf = kMlpN4;
    g.err = L.err;
    if ((rc = gemm_bf16(in, kMlpH, m->w.w4t, kMlpH, g, st))) return rc;
    cudaMemsetAsync(L.fb_count, 0, sizeof(int), st);
    ApplyArgs p{};
    p.y = L.y; p.env = L.env; p.norm = m->norm_d; p.n0 = n0; p.cnt = cnt; p.resid_tol = resid_tol;
    p.fb_list = L.fb_list; p.fb_count = L.fb_count; p.fb_cap = L.chunk; p.stats = L.stats;
    k_mlp_apply<<<(cnt + 127) / 128, 128, 0, st>>>(a, p);
    k_micro_src_list<<<148 * 4, 128, 0, st>>>(a, n0, L.fb_list, L.fb_count, L.chunk);
    *launches += 7;
    if (cudaGetLastError() != cudaSuccess) return CRESS_E_CUDA;
  }
  launch_fall(a, st);
  *launches += a.defer_adjstni ? 1 : 2;
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

// s_cloudphy with the MLP in place of the process rates, fused: one
// persistent kernel over all cells (features, 4 GEMMs, application), the
// plain process rates on the rejected cells, the plain sedimentation.
int launch_cloudphy_fused(const MicroArgs& a, const float* w, Mlp* m, const LearnedBuffers& L, float resid_tol,
                          cudaStream_t st, long long* launches) {
  k_init_dtp<<<1, 1, 0, st>>>(a.dtp_bits, a.dtb);
  FusedMaps maps;
  int rc;
  if ((rc = encode_bf16_map(&maps.w1, m->w.w1t, kMlpH, kMlpK1, kMlpK1, 128)) ||
      (rc = encode_bf16_map(&maps.w2, m->w.w2t, kMlpH, kMlpH, kMlpH, 128)) ||
      (rc = encode_bf16_map(&maps.w3, m->w.w3t, kMlpH, kMlpH, kMlpH, 128)) ||
      (rc = encode_bf16_map(&maps.w4, m->w.w4t, kMlpN4, kMlpH, kMlpH, kMlpN4)))
    return rc;
  if (cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmem) != cudaSuccess)
    return CRESS_E_CUDA;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  FusedArgs p{};
  p.w = w;
  p.norm = m->norm_d;
  p.params = m->params;
  p.ncell = (long long)(a.g.ni - 3) * (a.g.nj - 3) * (a.g.nk - 1);
  p.resid_tol = resid_tol;
  p.fb_list = L.fb_list;
  p.fb_count = L.fb_count;
  p.fb_cap = L.chunk;
  p.stats = L.stats;
  p.err = L.err;
  cudaMemsetAsync(L.fb_count, 0, sizeof(int), st);
  const long long ntiles = (p.ncell + kFusedTile - 1) / kFusedTile;
  const int grid = (int)(ntiles < 2 * nsm ? ntiles : 2 * nsm);   // two blocks per SM
  k_mlp_fused<<<grid, kFusedThreads, kFusedSmem, st>>>(maps, a, p);
  k_micro_src_list<<<nsm * 4, 128, 0, st>>>(a, 0, L.fb_list, L.fb_count, L.chunk);
  launch_fall(a, st);
  *launches += a.defer_adjstni ? 4 : 5;
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress
