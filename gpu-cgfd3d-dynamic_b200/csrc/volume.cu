// volume.cu -- fused volume stage kernels.
//
// One RK stage of every grid point outside the split-node slabs of the
// faults: right-hand side of the velocity-stress system and the stage's
// Runge-Kutta update in one pass.
//   * interior stencil   sv_curv_col_el_iso_rhs_inner_gpu
//                        (src/forward/sv_curv_col_el_iso_gpu.cu:232-388)
//   * traction image     sv_curv_col_el_iso_rhs_timg_z2_gpu  (:399-600)
//   * velocity below the free surface
//                        sv_curv_col_el_iso_rhs_vlow_z2_gpu  (:607-747)
//   * CFS-PML correction and auxiliary-field RHS
//                        sv_curv_col_el_iso_rhs_cfspml_gpu   (:825-1290)
//   * RK stage update    wav_update / wav_update_end (src/forward/wav_t.cu:219-234)
//                        and the PML auxiliary updates of drv_rk_curv_col.cu:329-568
// The reference runs these as 9-10 launches per stage plus three full
// read-modify-write sweeps of the wavefield for the RK update.  Here the
// domain is cut into boxes: the interior box (no PML, no surface rows) runs
// k_volume<INTERIOR>, whose code holds no boundary logic, and the shell of
// PML slabs and the top four rows runs k_volume<SHELL>.  Each stage reads
// the input level (stencil halos come from L1/L2), the metric and the medium
// once and writes the output levels once.
//
// Roofline: HBM-bound.  Algorithmic traffic per point and step is
// 192 floats = 768 B (21+18, 39+18, 39+18, 30+9 floats over the 4 stages).
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

constexpr int BX = 32, BY = 8;

// conservative traction J * (e . sigma_row) at point q for metric row `ax`
// (MXIX, METX or MZTX) and stress row r (0: xx,xy,xz; 1: xy,yy,yz;
// 2: xz,yz,zz)
__device__ __forceinline__ float ctrac(const float *__restrict__ w, const float *__restrict__ met,
                                       long sc, long q, int ax, int r) {
  const int c0 = r == 0 ? TXX : (r == 1 ? TXY : TXZ);
  const int c1 = r == 0 ? TXY : (r == 1 ? TYY : TYZ);
  const int c2 = r == 0 ? TXZ : (r == 1 ? TYZ : TZZ);
  return __ldg(met + MJAC * sc + q) * (__ldg(met + ax * sc + q) * __ldg(w + c0 * sc + q) +
                                       __ldg(met + (ax + 1) * sc + q) * __ldg(w + c1 * sc + q) +
                                       __ldg(met + (ax + 2) * sc + q) * __ldg(w + c2 * sc + q));
}

// Accumulate one direction's derivatives straight into the velocity
// gradient G[c][b] = dV_c/dx_b and the momentum sums
// s_r = sum_a e_a . d(sigma_row r)/dxi_a, so that only 12 accumulators stay
// live instead of 27 derivatives.
template <int F>
__device__ __forceinline__ void acc_vel(const float *__restrict__ w, long sc, long st, const float ea[3],
                                        float G[3][3], float dv[3]) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float d = drp<F>(w + (VX + c) * sc, st);
    dv[c] = d;
    G[c][0] += ea[0] * d; G[c][1] += ea[1] * d; G[c][2] += ea[2] * d;
  }
}
template <int F>
__device__ __forceinline__ void acc_stress(const float *__restrict__ w, long sc, long st, const float ea[3],
                                           float s[3]) {
  float d;
  d = drp<F>(w + TXX * sc, st); s[0] += ea[0] * d;
  d = drp<F>(w + TYY * sc, st); s[1] += ea[1] * d;
  d = drp<F>(w + TZZ * sc, st); s[2] += ea[2] * d;
  d = drp<F>(w + TYZ * sc, st); s[1] += ea[2] * d; s[2] += ea[1] * d;
  d = drp<F>(w + TXZ * sc, st); s[0] += ea[2] * d; s[2] += ea[0] * d;
  d = drp<F>(w + TXY * sc, st); s[0] += ea[1] * d; s[1] += ea[0] * d;
}

__device__ __forceinline__ void hooke(const float G[3][3], float lam, float mu, float l2m, float h[9]) {
  h[TXX] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]);
  h[TYY] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]);
  h[TZZ] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]);
  h[TXY] = mu * (G[0][1] + G[1][0]);
  h[TXZ] = mu * (G[0][2] + G[2][0]);
  h[TYZ] = mu * (G[1][2] + G[2][1]);
}

template <int MODE>
__device__ __forceinline__ void rk_update(const VolArgs &a, long p, const float h[9]) {
  const long sc = a.g.scmp;
#pragma unroll
  for (int c = 0; c < 9; c++) {
    const long o = c * sc + p;
    if (MODE == RK_FIRST) {
      const float v = __ldg(a.cur + o);
      a.out[o] = v + a.ca * h[c];
      a.end[o] = v + a.cb * h[c];
    } else if (MODE == RK_MID) {
      a.out[o] = __ldg(a.pre + o) + a.ca * h[c];
      a.end[o] += a.cb * h[c];
    } else {
      a.end[o] += a.cb * h[c];
    }
  }
}

enum { INTERIOR = 0, SHELL = 1 };

template <int ID, int JD, int KD, int MODE, int KIND>
__global__ void __launch_bounds__(BX * BY, KIND == INTERIOR ? 3 : 2) k_volume(const VolArgs a) {
  const Grid &g = a.g;
  // locate the box of this block
  int b = 0;
#pragma unroll 1
  while (b + 1 < a.nbox && (int)blockIdx.x >= a.box[b + 1].first) b++;
  const VolBox &B = a.box[b];
  const int bid = blockIdx.x - B.first;
  const int bx = bid % B.nbx, rem = bid / B.nbx, by = rem % B.nby, bz = rem / B.nby;
  const int i = B.i0 + bx * BX + threadIdx.x;
  const int j = B.j0 + by * BY + threadIdx.y;
  const int k = B.k0 + bz;
  if (i > B.i1 || j > B.j1) return;
  const int I = i + NG, J = j + NG, K = k + NG;
  // split-node slabs (i0-3..i0+3 of unwelded nodes) belong to the fault kernels
  for (int f = 0; f < a.nfault; f++) {
    const int d = I - a.fi0[f];
    if (d >= -3 && d <= 3 && (__ldg(a.fflag[f] + J + (long)K * g.ny) & FL_SPLIT)) return;
  }
  const long p = g.at(I, J, K);
  const long sy = g.sy, sz = g.sz, sc = g.scmp;
  const float *__restrict__ w = a.cur + p;
  float e[3][3];
#pragma unroll
  for (int q = 0; q < 9; q++) e[q / 3][q % 3] = __ldg(a.met + (1 + q) * sc + p);
  const float lam = __ldg(a.med + p), mu = __ldg(a.med + sc + p), slw = __ldg(a.med + 2 * sc + p);
  const float l2m = lam + 2.0f * mu;

  float h[9];
  float G[3][3] = { { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f } };
  float s[3] = { 0.f, 0.f, 0.f };
  float dvx[3], dvy[3], dvz[3];
  acc_vel<ID>(w, sc, 1, e[0], G, dvx);
  acc_stress<ID>(w, sc, 1, e[0], s);
  acc_vel<JD>(w, sc, sy, e[1], G, dvy);
  acc_stress<JD>(w, sc, sy, e[1], s);
  acc_stress<KD>(w, sc, sz, e[2], s);
  if (KIND == INTERIOR) {
    acc_vel<KD>(w, sc, sz, e[2], G, dvz);
    h[VX] = slw * s[0]; h[VY] = slw * s[1]; h[VZ] = slw * s[2];
    hooke(G, lam, mu, l2m, h);
    rk_update<MODE>(a, p, h);
    return;
  }

  // ---- shell: PML slabs and the rows under the free surface ----------------
  const int nk2 = g.nk + NG - 1;
  const bool vlow = a.isfree && K >= nk2 - 2;
  if (!vlow) {
    acc_vel<KD>(w, sc, sz, e[2], G, dvz);
    hooke(G, lam, mu, l2m, h);
  } else {
    // velocity gradient below the surface: conversion matrices at the
    // surface, 2nd / 4th order one-sided dz one and two rows below
    float dz[3];
    if (K == nk2) {
      const float *X = a.free_mat + ((long)J * g.nx + I) * 9;
      const float *Y = X + (long)g.ny * g.nx * 9;
      float o1[3], o2[3];
      mv3(X, dvx, o1); mv3(Y, dvy, o2);
      dz[0] = o1[0] + o2[0]; dz[1] = o1[1] + o2[1]; dz[2] = o1[2] + o2[2];
    } else if (K == nk2 - 1) {
      dz[0] = mac22(w + VX * sc, sz, KD); dz[1] = mac22(w + VY * sc, sz, KD); dz[2] = mac22(w + VZ * sc, sz, KD);
    } else {
      dz[0] = mac24(w + VX * sc, sz, KD); dz[1] = mac24(w + VY * sc, sz, KD); dz[2] = mac24(w + VZ * sc, sz, KD);
    }
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int bb = 0; bb < 3; bb++) G[c][bb] += e[2][bb] * dz[c];
    hooke(G, lam, mu, l2m, h);
  }
  h[VX] = slw * s[0]; h[VY] = slw * s[1]; h[VZ] = slw * s[2];
  if (a.isfree && K >= nk2 - (KD ? 3 : 1)) {
    // traction image on the momentum equation in the top rows
    const float *cur = a.cur;
    const float sj = slw / __ldg(a.met + MJAC * sc + p);
#pragma unroll 1
    for (int r = 0; r < 3; r++) {
      float dx = 0.f, dy = 0.f, dzz = 0.f;
#pragma unroll
      for (int n = 0; n < 5; n++) {
        const int o = ID ? n - 1 : n - 3;
        dx += drp_w(ID, n) * ctrac(cur, a.met, sc, p + o, MXIX, r);
      }
#pragma unroll
      for (int n = 0; n < 5; n++) {
        const int o = JD ? n - 1 : n - 3;
        dy += drp_w(JD, n) * ctrac(cur, a.met, sc, p + o * sy, METX, r);
      }
#pragma unroll
      for (int n = 0; n < 5; n++) {
        const int kk = K + (KD ? n - 1 : n - 3);
        float v = 0.f;
        if (kk < nk2) v = ctrac(cur, a.met, sc, g.at(I, J, kk), MZTX, r);
        else if (kk > nk2) v = -ctrac(cur, a.met, sc, g.at(I, J, 2 * nk2 - kk), MZTX, r);
        dzz += drp_w(KD, n) * v;
      }
      h[VX + r] = (dx + dy + dzz) * sj;
    }
  }

  // CFS-PML: faces add up where they overlap
#pragma unroll
  for (int fc = 0; fc < 6; fc++) {
    const int d = fc >> 1;
    const PmlFaceDev &P = a.pml[fc];
    if (!P.on) continue;
    const int li = I - P.i1, lj = J - P.j1, lk = K - P.k1;
    if (li < 0 || li >= P.fni || lj < 0 || lj >= P.fnj || lk < 0 || lk >= P.fnk) continue;
    const int layer = d == 0 ? li : (d == 1 ? lj : lk);
    const float cA = __ldg(P.A + layer), cB = __ldg(P.B + layer), cD = __ldg(P.D + layer);
    const float ex = e[d][0], ey = e[d][1], ez = e[d][2];
    const int DF = d == 0 ? ID : (d == 1 ? JD : KD);
    const long st = d == 0 ? 1 : (d == 1 ? sy : sz);
    float Dd[9];
#pragma unroll
    for (int c = 0; c < 9; c++) Dd[c] = DF ? drp<1>(w + c * sc, st) : drp<0>(w + c * sc, st);
    float r[9];
    r[VX] = slw * (ex * Dd[TXX] + ey * Dd[TXY] + ez * Dd[TXZ]);
    r[VY] = slw * (ex * Dd[TXY] + ey * Dd[TYY] + ez * Dd[TYZ]);
    r[VZ] = slw * (ex * Dd[TXZ] + ey * Dd[TYZ] + ez * Dd[TZZ]);
    r[TXX] = l2m * ex * Dd[VX] + lam * ey * Dd[VY] + lam * ez * Dd[VZ];
    r[TYY] = lam * ex * Dd[VX] + l2m * ey * Dd[VY] + lam * ez * Dd[VZ];
    r[TZZ] = lam * ex * Dd[VX] + lam * ey * Dd[VY] + l2m * ez * Dd[VZ];
    r[TXY] = mu * (ey * Dd[VX] + ex * Dd[VY]);
    r[TXZ] = mu * (ez * Dd[VX] + ex * Dd[VZ]);
    r[TYZ] = mu * (ez * Dd[VY] + ey * Dd[VZ]);
    const long pa = li + (long)lj * P.fni + (long)lk * P.fni * P.fnj;
    const float *ac = P.acur + pa;
    float ar[9];
#pragma unroll
    for (int c = 0; c < 9; c++) {
      const float av = __ldg(ac + c * P.siz);
      h[c] += (cB - 1.0f) * r[c] - cB * av;
      ar[c] = cD * r[c] - cA * av;
    }
    if (d < 2 && a.isfree && K == nk2) {
      // free-surface coupling of the x / y faces: the d-derivative of the
      // surface-converted dz velocity gradient
      const float *X = a.free_mat + (long)(d == 0 ? 0 : 1) * g.ny * g.nx * 9 + ((long)J * g.nx + I) * 9;
      const float dd[3] = { Dd[VX], Dd[VY], Dd[VZ] };
      float z[3];
      mv3(X, dd, z);
      const float zx = e[2][0], zy = e[2][1], zz = e[2][2];
      float q[9];
      q[TXX] = l2m * (zx * z[0]) + lam * (zy * z[1] + zz * z[2]);
      q[TYY] = l2m * (zy * z[1]) + lam * (zx * z[0] + zz * z[2]);
      q[TZZ] = l2m * (zz * z[2]) + lam * (zx * z[0] + zy * z[1]);
      q[TXY] = mu * (zy * z[0] + zx * z[1]);
      q[TXZ] = mu * (zz * z[0] + zx * z[2]);
      q[TYZ] = mu * (zz * z[1] + zy * z[2]);
#pragma unroll
      for (int c = TXX; c <= TXY; c++) { h[c] += (cB - 1.0f) * q[c]; ar[c] += cD * q[c]; }
    }
    float *aE = P.aend + pa;
#pragma unroll
    for (int c = 0; c < 9; c++) {
      const long o = c * P.siz;
      if (MODE == RK_FIRST) {
        const float av = __ldg(ac + o);
        P.aout[pa + o] = av + a.ca * ar[c];
        aE[o] = av + a.cb * ar[c];
      } else if (MODE == RK_MID) {
        P.aout[pa + o] = __ldg(P.apre + pa + o) + a.ca * ar[c];
        aE[o] += a.cb * ar[c];
      } else {
        aE[o] += a.cb * ar[c];
      }
    }
  }
  rk_update<MODE>(a, p, h);
}

template <int ID, int JD, int KD, int KIND>
void launch4(const VolArgs &a, int mode, cudaStream_t st) {
  if (a.nbox == 0) return;
  const dim3 blk(BX, BY, 1);
  const dim3 grd(a.nblocks);
  if (mode == RK_FIRST) k_volume<ID, JD, KD, RK_FIRST, KIND><<<grd, blk, 0, st>>>(a);
  else if (mode == RK_MID) k_volume<ID, JD, KD, RK_MID, KIND><<<grd, blk, 0, st>>>(a);
  else k_volume<ID, JD, KD, RK_LAST, KIND><<<grd, blk, 0, st>>>(a);
}

template <int KIND>
void launch_kind(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  switch (idir * 4 + jdir * 2 + kdir) {
    case 0: launch4<0, 0, 0, KIND>(a, mode, st); break;
    case 1: launch4<0, 0, 1, KIND>(a, mode, st); break;
    case 2: launch4<0, 1, 0, KIND>(a, mode, st); break;
    case 3: launch4<0, 1, 1, KIND>(a, mode, st); break;
    case 4: launch4<1, 0, 0, KIND>(a, mode, st); break;
    case 5: launch4<1, 0, 1, KIND>(a, mode, st); break;
    case 6: launch4<1, 1, 0, KIND>(a, mode, st); break;
    default: launch4<1, 1, 1, KIND>(a, mode, st); break;
  }
}

}  // namespace

// boxes (interior indices, inclusive) -> block layout of one launch
void volume_boxes(VolArgs &a, const int (*boxes)[6], int n) {
  a.nbox = 0;
  int first = 0;
  for (int q = 0; q < n; q++) {
    const int *b = boxes[q];
    if (b[1] < b[0] || b[3] < b[2] || b[5] < b[4]) continue;
    VolBox &B = a.box[a.nbox++];
    B.i0 = b[0]; B.i1 = b[1]; B.j0 = b[2]; B.j1 = b[3]; B.k0 = b[4];
    B.nbx = (b[1] - b[0] + BX) / BX;
    B.nby = (b[3] - b[2] + BY) / BY;
    B.first = first;
    first += B.nbx * B.nby * (b[5] - b[4] + 1);
  }
  a.nblocks = first;
}

void launch_volume(const VolArgs &interior, const VolArgs &shell, int idir, int jdir, int kdir, int mode,
                   cudaStream_t st) {
  launch_kind<INTERIOR>(interior, idir, jdir, kdir, mode, st);
  launch_kind<SHELL>(shell, idir, jdir, kdir, mode, st);
}

}  // namespace cgfd
