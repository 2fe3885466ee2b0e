// ops.cuh -- finite-difference operators of the MacCormack/DRP scheme
// (src/forward/fd_t.h:9-140, tables in src/forward/fd_t.cu:64-110) as
// sm_100a device functions, plus the argument blocks of the stage kernels.
#pragma once
#include <cuda_runtime.h>

#include "../../include/cgfd.h"
#include "common.h"

namespace cgfd {

// one-sided 5-point DRP derivative, forward (F = 1: offsets -1..3) or
// backward (F = 0: offsets -3..1)
constexpr real kC1 = RL(-0.291647047), kC2 = RL(-0.666745142), kC3 = RL(1.250117713),
               kC4 = RL(-0.333411808), kC5 = RL(0.041686285);
// 2-point and 3-point one-sided operators (MAC22, MAC24)
constexpr real kB1 = RL(-7.0) / RL(6.0), kB2 = RL(8.0) / RL(6.0), kB3 = RL(-1.0) / RL(6.0);
// one-sided traction-image weights at split nodes
constexpr real kA0 = RL(1.2500392377), kA1 = RL(1.5417647610), kA2 = RL(-0.3334118088),
               kA3 = RL(0.0416862855);

template <int F>
__device__ __forceinline__ real drp(const real *__restrict__ p, long s) {
  if (F)
    return kC1 * __ldg(p - s) + kC2 * __ldg(p) + kC3 * __ldg(p + s) + kC4 * __ldg(p + 2 * s) + kC5 * __ldg(p + 3 * s);
  else
    return -(kC1 * __ldg(p + s) + kC2 * __ldg(p) + kC3 * __ldg(p - s) + kC4 * __ldg(p - 2 * s) + kC5 * __ldg(p - 3 * s));
}
__device__ __forceinline__ real drp_rt(const real *p, long s, int f) {
  return f ? drp<1>(p, s) : drp<0>(p, s);
}
__device__ __forceinline__ real mac22(const real *p, long s, int f) {
  return f ? (__ldg(p + s) - __ldg(p)) : (__ldg(p) - __ldg(p - s));
}
__device__ __forceinline__ real mac24(const real *p, long s, int f) {
  return f ? (kB1 * __ldg(p) + kB2 * __ldg(p + s) + kB3 * __ldg(p + 2 * s))
           : -(kB1 * __ldg(p) + kB2 * __ldg(p - s) + kB3 * __ldg(p - 2 * s));
}
// DRP on register values v[-3..3] centred at v
__device__ __forceinline__ real drp_v(const real *v, int f) {
  return f ? (kC1 * v[-1] + kC2 * v[0] + kC3 * v[1] + kC4 * v[2] + kC5 * v[3])
           : -(kC1 * v[1] + kC2 * v[0] + kC3 * v[-1] + kC4 * v[-2] + kC5 * v[-3]);
}

// offsets of the DRP stencil in table order and the matching weights
__device__ __forceinline__ int drp_off(int f, int n) { return f ? n - 1 : n - 3; }
__device__ __forceinline__ real drp_w(int f, int n) {
  const real wf[5] = { kC1, kC2, kC3, kC4, kC5 };
  return f ? wf[n] : -wf[4 - n];
}

__device__ __forceinline__ void mv3(const real *__restrict__ m, const real *v, real *o) {
  o[0] = __ldg(m + 0) * v[0] + __ldg(m + 1) * v[1] + __ldg(m + 2) * v[2];
  o[1] = __ldg(m + 3) * v[0] + __ldg(m + 4) * v[1] + __ldg(m + 5) * v[2];
  o[2] = __ldg(m + 6) * v[0] + __ldg(m + 7) * v[1] + __ldg(m + 8) * v[2];
}

// level slots
enum { LP = 0, LA = 1, LB = 2, LE = 3 };
// RK mode of a stage: first (out tmp & end from P), middle, last
enum { RK_FIRST = 0, RK_MID = 1, RK_LAST = 2 };

// a box of interior points (inclusive bounds) covered by one launch;
// blocks [first, next box's first) belong to it
struct VolBox {
  int i0, i1, j0, j1, k0, k1;
  int nbx, nby, first;
};

struct VolArgs {
  Grid g;
  int nbox, nblocks;
  int ychunk;                  // interior kernel: y tiles per chunk (z marches within a chunk)
  VolBox box[16];
  const real *cur, *pre;
  real *out, *end;            // next-stage level (null at the last stage), E
  const real *coef, *free_mat;   // packed metric and medium (coef_row / coef_jac)
  real ca, cb;
  int isfree;
  int nfault;
  // 1: the interior kernel leaves the fault planes x = i0 within each
  // fault's split box grown by 3 nodes (welded nodes too; ghost-inclusive
  // J0, J1, K0, K1 in fdef) to a later launch, so that it reads nothing the
  // stage's first fault kernels write and may run beside them; outside that
  // box no tap of a plane point reaches a split node
  int defer_i0;
  int fi0[MAXF];
  int fdef[MAXF][4];
  const uint8_t *fflag[MAXF];
  PmlFaceDev pml[6];           // indexed 2*dim + side; `on` = 0 when absent
};

struct FaultArgs {
  Grid g;
  FaultDev F;
  const real *wcur, *wpre;
  real *wout, *wend;
  const real *coef, *free_mat;   // packed metric and medium (coef_row / coef_jac)
  // fault wavefield levels [9][2 sides][ny*nz]: stage input, time-n level,
  // next-stage output (null at the last stage), end accumulator
  const real *fc, *fp;
  real *fo, *fe;
  int idir, jdir, kdir;
  int mode;
  real ca, cb, rkb, dt;
  int isfree, imethod;
  int j0, k0, nj, nk;          // launch box of split nodes (interior indices)
  // welded nodes whose fault fields a stage reads (the split box grown by
  // the 3-node stencil reach, or the whole plane without split nodes)
  int wj0, wk0, wnj, wnk;
  Ctl *ctl;
  // tractions J e_a . sigma of the stage input at x = i0-6..i0-1, i0+1..i0+6
  // over the split box grown by 3 nodes in j and k: [12][9][tnk][tnj],
  // components T1 (e_xi), T2 (e_eta), T3 (e_zeta); T2 and T3 only for
  // |x - i0| <= 3.  tj0 / tk0: ghost-inclusive j / k of element (0, 0).
  real *trac;
  int tj0, tk0, tnj, tnk;
};

struct StationArgs {
  Grid g;
  StationDev st;
  const real *w;
  const real *fout[MAXF];
  long ns;
  Ctl *ctl;
};

// exponential sponge on the end-of-step level: masks E[nx | ny | nz]
// (ghost-inclusive index), blocks of ghost-inclusive inclusive bounds
// i1 i2 j1 j2 k1 k2, first[b] = points of the blocks before b
struct SpongeArgs {
  Grid g;
  real *w;
  const real *E;
  int nblk;
  int blk[6][6];
  long first[7];
};

// peak ground motion of the free surface: end-of-step and time-n levels,
// peaks [15][nj][ni] and displacement [3][nj][ni] at interior (i, j)
struct PeakArgs {
  Grid g;
  const real *wend, *wpre;
  real *pg, *dis;
  real dt;
};

}  // namespace cgfd
