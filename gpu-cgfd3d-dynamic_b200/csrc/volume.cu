// volume.cu -- fused volume stage kernel.
//
// One launch per RK stage computes, for every grid point outside the
// split-node slabs of the faults, the right-hand side of the velocity-stress
// system and applies the stage's Runge-Kutta update in the same pass:
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
// read-modify-write sweeps of the wavefield for the RK update; here each
// stage reads the input level (with stencil halos), the metric and the
// medium once and writes the output levels once.
//
// Roofline: HBM-bound.  Algorithmic traffic per point and step is
// 192 floats = 768 B (21+18, 39+18, 39+18, 30+9 floats over the 4 stages).
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

// conservative traction J * (e . sigma_row) at point q for metric row `ax`
// (1 = xi, 4 = eta, 7 = zeta) and stress row r (0: xx,xy,xz; 1: xy,yy,yz;
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

template <int ID, int JD, int KD, int MODE>
__global__ void __launch_bounds__(256) k_volume(const VolArgs a) {
  const Grid &g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.ni || j >= g.nj) return;
  const int I = i + NG, J = j + NG, K = k + NG;
  // split-node slabs (i0-3..i0+3 of unwelded nodes) belong to the fault kernels
  for (int f = 0; f < a.nfault; f++) {
    const int d = I - a.fi0[f];
    if (d >= -3 && d <= 3 && (__ldg(a.fflag[f] + J + (long)K * g.ny) & FL_SPLIT)) return;
  }
  const long p = g.at(I, J, K);
  const long sy = g.sy, sz = g.sz, sc = g.scmp;
  const float *__restrict__ w = a.cur + p;

  float D[3][9];
#pragma unroll
  for (int c = 0; c < 9; c++) {
    D[0][c] = drp<ID>(w + c * sc, 1);
    D[1][c] = drp<JD>(w + c * sc, sy);
    D[2][c] = drp<KD>(w + c * sc, sz);
  }
  float e[3][3];
#pragma unroll
  for (int q = 0; q < 9; q++) e[q / 3][q % 3] = __ldg(a.met + (1 + q) * sc + p);
  const float lam = __ldg(a.med + p), mu = __ldg(a.med + sc + p), slw = __ldg(a.med + 2 * sc + p);
  const float l2m = lam + 2.0f * mu;

  float h[9];
  {
    // momentum: rho dV_r/dt = sum_a e_a . d(sigma_row r)/dxi_a
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      s0 += e[ax][0] * D[ax][TXX] + e[ax][1] * D[ax][TXY] + e[ax][2] * D[ax][TXZ];
      s1 += e[ax][0] * D[ax][TXY] + e[ax][1] * D[ax][TYY] + e[ax][2] * D[ax][TYZ];
      s2 += e[ax][0] * D[ax][TXZ] + e[ax][1] * D[ax][TYZ] + e[ax][2] * D[ax][TZZ];
    }
    h[VX] = slw * s0; h[VY] = slw * s1; h[VZ] = slw * s2;
  }
  // Hooke: velocity gradient G[c][b] = dV_c/dx_b = sum_a e_a[b] dV_c/dxi_a
  auto hooke = [&](const float dvx[3], const float dvy[3], const float dvz[3]) {
    float G[3][3];
#pragma unroll
    for (int b = 0; b < 3; b++) {
      G[0][b] = e[0][b] * dvx[0] + e[1][b] * dvx[1] + e[2][b] * dvx[2];
      G[1][b] = e[0][b] * dvy[0] + e[1][b] * dvy[1] + e[2][b] * dvy[2];
      G[2][b] = e[0][b] * dvz[0] + e[1][b] * dvz[1] + e[2][b] * dvz[2];
    }
    h[TXX] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]);
    h[TYY] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]);
    h[TZZ] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]);
    h[TXY] = mu * (G[0][1] + G[1][0]);
    h[TXZ] = mu * (G[0][2] + G[2][0]);
    h[TYZ] = mu * (G[1][2] + G[2][1]);
  };
  {
    const float dvx[3] = { D[0][VX], D[1][VX], D[2][VX] };
    const float dvy[3] = { D[0][VY], D[1][VY], D[2][VY] };
    const float dvz[3] = { D[0][VZ], D[1][VZ], D[2][VZ] };
    hooke(dvx, dvy, dvz);
  }

  const int nk2 = g.nk + NG - 1;
  if (a.isfree && K >= nk2 - 3) {
    // traction image on the momentum equation in the top layers
    if (K >= nk2 - (KD ? 3 : 1)) {
      const float *cur = a.cur;
      const float sj = slw / __ldg(a.met + MJAC * sc + p);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        float dx = 0.f, dy = 0.f, dz = 0.f;
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
          dz += drp_w(KD, n) * v;
        }
        h[VX + r] = (dx + dy + dz) * sj;
      }
    }
    // velocity gradient below the surface: conversion matrices at the
    // surface, 2nd / 4th order one-sided dz one and two points below
    if (K >= nk2 - 2) {
      float dz[3];
      if (K == nk2) {
        const float *X = a.free_mat + ((long)J * g.nx + I) * 9;
        const float *Y = X + (long)g.ny * g.nx * 9;
        const float dx3[3] = { D[0][VX], D[0][VY], D[0][VZ] }, dy3[3] = { D[1][VX], D[1][VY], D[1][VZ] };
        float o1[3], o2[3];
        mv3(X, dx3, o1); mv3(Y, dy3, o2);
        dz[0] = o1[0] + o2[0]; dz[1] = o1[1] + o2[1]; dz[2] = o1[2] + o2[2];
      } else if (K == nk2 - 1) {
        dz[0] = mac22(w + VX * sc, sz, KD); dz[1] = mac22(w + VY * sc, sz, KD); dz[2] = mac22(w + VZ * sc, sz, KD);
      } else {
        dz[0] = mac24(w + VX * sc, sz, KD); dz[1] = mac24(w + VY * sc, sz, KD); dz[2] = mac24(w + VZ * sc, sz, KD);
      }
      const float dvx[3] = { D[0][VX], D[1][VX], dz[0] };
      const float dvy[3] = { D[0][VY], D[1][VY], dz[1] };
      const float dvz[3] = { D[0][VZ], D[1][VZ], dz[2] };
      hooke(dvx, dvy, dvz);
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
    float r[9];
    r[VX] = slw * (ex * D[d][TXX] + ey * D[d][TXY] + ez * D[d][TXZ]);
    r[VY] = slw * (ex * D[d][TXY] + ey * D[d][TYY] + ez * D[d][TYZ]);
    r[VZ] = slw * (ex * D[d][TXZ] + ey * D[d][TYZ] + ez * D[d][TZZ]);
    r[TXX] = l2m * ex * D[d][VX] + lam * ey * D[d][VY] + lam * ez * D[d][VZ];
    r[TYY] = lam * ex * D[d][VX] + l2m * ey * D[d][VY] + lam * ez * D[d][VZ];
    r[TZZ] = lam * ex * D[d][VX] + lam * ey * D[d][VY] + l2m * ez * D[d][VZ];
    r[TXY] = mu * (ey * D[d][VX] + ex * D[d][VY]);
    r[TXZ] = mu * (ez * D[d][VX] + ex * D[d][VZ]);
    r[TYZ] = mu * (ez * D[d][VY] + ey * D[d][VZ]);
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
      const float dd[3] = { D[d][VX], D[d][VY], D[d][VZ] };
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

  // RK stage update
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

template <int ID, int JD, int KD>
void launch3(const VolArgs &a, int mode, cudaStream_t st) {
  dim3 blk(32, 8, 1);
  dim3 grd((a.g.ni + 31) / 32, (a.g.nj + 7) / 8, a.g.nk);
  if (mode == RK_FIRST) k_volume<ID, JD, KD, RK_FIRST><<<grd, blk, 0, st>>>(a);
  else if (mode == RK_MID) k_volume<ID, JD, KD, RK_MID><<<grd, blk, 0, st>>>(a);
  else k_volume<ID, JD, KD, RK_LAST><<<grd, blk, 0, st>>>(a);
}

}  // namespace

void launch_volume(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  const int key = idir * 4 + jdir * 2 + kdir;
  switch (key) {
    case 0: launch3<0, 0, 0>(a, mode, st); break;
    case 1: launch3<0, 0, 1>(a, mode, st); break;
    case 2: launch3<0, 1, 0>(a, mode, st); break;
    case 3: launch3<0, 1, 1>(a, mode, st); break;
    case 4: launch3<1, 0, 0>(a, mode, st); break;
    case 5: launch3<1, 0, 1>(a, mode, st); break;
    case 6: launch3<1, 1, 0>(a, mode, st); break;
    default: launch3<1, 1, 1>(a, mode, st); break;
  }
}

}  // namespace cgfd
