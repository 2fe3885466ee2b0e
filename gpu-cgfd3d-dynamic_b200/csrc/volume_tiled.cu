// volume_tiled.cu -- z-marching, shared-memory tiled volume stage kernel.
//
// Same operator as volume.cu (inner stencil + traction image + velocity-low
// rows + CFS-PML + RK stage update, sv_curv_col_el_iso_gpu.cu:232-1290 and
// wav_t.cu:219-234), organised for HBM:
//   * a block owns a 32 x 8 column of (x, y) points and marches up a chunk
//     of z rows;
//   * each thread keeps the five z samples the one-sided z operator needs of
//     all nine components in registers (a queue shifted per row), so a row
//     costs one coalesced load per component for z;
//   * the nine components of the current row are staged in shared memory
//     with the one-sided x / y halo of this stage's operator direction, so
//     x and y derivatives read shared memory instead of L1/L2;
//   * the RHS is built direction by direction; the CFS-PML correction of a
//     face with normal d is formed from direction d's part right away.
// Algorithmic HBM traffic per point and step: 192 floats = 768 B.
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

constexpr int TX = 32, TY = 8;

__device__ __forceinline__ float ctrac_t(const float *__restrict__ w, const float *__restrict__ met,
                                         long sc, long q, int ax, int r) {
  const int c0 = r == 0 ? TXX : (r == 1 ? TXY : TXZ);
  const int c1 = r == 0 ? TXY : (r == 1 ? TYY : TYZ);
  const int c2 = r == 0 ? TXZ : (r == 1 ? TYZ : TZZ);
  return __ldg(met + MJAC * sc + q) * (__ldg(met + ax * sc + q) * __ldg(w + c0 * sc + q) +
                                       __ldg(met + (ax + 1) * sc + q) * __ldg(w + c1 * sc + q) +
                                       __ldg(met + (ax + 2) * sc + q) * __ldg(w + c2 * sc + q));
}

template <int F>
__device__ __forceinline__ float wdrp(int n) {
  return F ? (n == 0 ? kC1 : n == 1 ? kC2 : n == 2 ? kC3 : n == 3 ? kC4 : kC5)
           : (n == 0 ? -kC5 : n == 1 ? -kC4 : n == 2 ? -kC3 : n == 3 ? -kC2 : -kC1);
}

// direction-d part of the RHS from the nine d-derivatives D[c] and e = e_d
__device__ __forceinline__ void rhs_dir(const float D[9], const float e[3], float lam, float mu, float l2m,
                                        float slw, float r[9]) {
  r[VX] = slw * (e[0] * D[TXX] + e[1] * D[TXY] + e[2] * D[TXZ]);
  r[VY] = slw * (e[0] * D[TXY] + e[1] * D[TYY] + e[2] * D[TYZ]);
  r[VZ] = slw * (e[0] * D[TXZ] + e[1] * D[TYZ] + e[2] * D[TZZ]);
  r[TXX] = l2m * e[0] * D[VX] + lam * (e[1] * D[VY] + e[2] * D[VZ]);
  r[TYY] = l2m * e[1] * D[VY] + lam * (e[0] * D[VX] + e[2] * D[VZ]);
  r[TZZ] = l2m * e[2] * D[VZ] + lam * (e[0] * D[VX] + e[1] * D[VY]);
  r[TXY] = mu * (e[1] * D[VX] + e[0] * D[VY]);
  r[TXZ] = mu * (e[2] * D[VX] + e[0] * D[VZ]);
  r[TYZ] = mu * (e[2] * D[VY] + e[1] * D[VZ]);
}

// PML face of normal d at this point (if any): add its correction to corr
// and advance its auxiliary fields
template <int MODE>
__device__ __forceinline__ void pml_face(const VolArgs &a, const PmlFaceDev &P, int d, int I, int J, int K,
                                         const float r[9], const float D[9], const float e2[3],
                                         float lam, float mu, float l2m, bool surf, long fidx, float corr[9]) {
  const int li = I - P.i1, lj = J - P.j1, lk = K - P.k1;
  if (li < 0 || li >= P.fni || lj < 0 || lj >= P.fnj || lk < 0 || lk >= P.fnk) return;
  const int layer = d == 0 ? li : (d == 1 ? lj : lk);
  const float cA = __ldg(P.A + layer), cB = __ldg(P.B + layer), cD = __ldg(P.D + layer);
  const long pa = li + (long)lj * P.fni + (long)lk * P.fni * P.fnj;
  float ar[9];
#pragma unroll
  for (int c = 0; c < 9; c++) {
    const float av = __ldg(P.acur + c * P.siz + pa);
    corr[c] += (cB - 1.0f) * r[c] - cB * av;
    ar[c] = cD * r[c] - cA * av;
  }
  if (surf) {
    // free-surface coupling of the x / y faces
    const float *X = a.free_mat + (long)(d == 0 ? 0 : 1) * a.g.ny * a.g.nx * 9 + fidx;
    const float dd[3] = { D[VX], D[VY], D[VZ] };
    float z[3];
    mv3(X, dd, z);
    float q[9];
    q[TXX] = l2m * (e2[0] * z[0]) + lam * (e2[1] * z[1] + e2[2] * z[2]);
    q[TYY] = l2m * (e2[1] * z[1]) + lam * (e2[0] * z[0] + e2[2] * z[2]);
    q[TZZ] = l2m * (e2[2] * z[2]) + lam * (e2[0] * z[0] + e2[1] * z[1]);
    q[TXY] = mu * (e2[1] * z[0] + e2[0] * z[1]);
    q[TXZ] = mu * (e2[2] * z[0] + e2[0] * z[2]);
    q[TYZ] = mu * (e2[2] * z[1] + e2[1] * z[2]);
#pragma unroll
    for (int c = TXX; c <= TXY; c++) { corr[c] += (cB - 1.0f) * q[c]; ar[c] += cD * q[c]; }
  }
#pragma unroll
  for (int c = 0; c < 9; c++) {
    const long o = c * P.siz + pa;
    if (MODE == RK_FIRST) {
      const float av = __ldg(P.acur + o);
      P.aout[o] = av + a.ca * ar[c];
      P.aend[o] = av + a.cb * ar[c];
    } else if (MODE == RK_MID) {
      P.aout[o] = __ldg(P.apre + o) + a.ca * ar[c];
      P.aend[o] += a.cb * ar[c];
    } else {
      P.aend[o] += a.cb * ar[c];
    }
  }
}

template <int ID, int JD, int KD, int MODE>
__global__ void __launch_bounds__(TX * TY, 2) k_volume_tiled(const VolArgs a) {
  constexpr int HXL = ID ? 1 : 3, HXR = ID ? 3 : 1;
  constexpr int HYL = JD ? 1 : 3, HYR = JD ? 3 : 1;
  constexpr int SX = TX + HXL + HXR, SY = TY + HYL + HYR;
  constexpr int M0 = KD ? 1 : 3;                 // queue slot of the current row
  constexpr int NHX = TY * (HXL + HXR), NHY = TX * (HYL + HYR), NH = NHX + NHY;
  __shared__ float tile[9][SY][SX];

  const Grid &g = a.g;
  const long sc = g.scmp, sy = g.sy;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = blockIdx.x * TX + tx, j = blockIdx.y * TY + ty;
  const int I = i + NG, J = j + NG;
  const bool inside = i < g.ni && j < g.nj;
  const bool valid = I < g.nx && J < g.ny;      // has a (ghost or interior) value
  const int kb = blockIdx.z * a.kchunk, ke = min(kb + a.kchunk, g.nk);
  const int nk2 = g.nk + NG - 1;
  const float *__restrict__ cur = a.cur;

  // slab of split nodes handled by the fault kernels
  int slab_f = -1;
  for (int f = 0; f < a.nfault; f++) {
    const int d = I - a.fi0[f];
    if (d >= -3 && d <= 3) slab_f = f;
  }

  float q[9][5];
  {
    const long p0 = valid ? g.at(I, J, kb + NG) : 0;
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const long o = p0 + (long)(KD ? m - 1 : m - 3) * g.sz;
#pragma unroll
      for (int c = 0; c < 9; c++) q[c][m] = valid ? __ldg(cur + c * sc + o) : 0.f;
    }
  }

  for (int k = kb; k < ke; k++) {
    const int K = k + NG;
    const long p = g.at(I, J, K);
    {
      const long o = p + (long)(KD ? 3 : 1) * g.sz;
#pragma unroll
      for (int c = 0; c < 9; c++) q[c][4] = valid ? __ldg(cur + c * sc + o) : 0.f;
    }
    // stage the row: own value from the queue, halo from global memory
#pragma unroll
    for (int c = 0; c < 9; c++) tile[c][ty + HYL][tx + HXL] = q[c][M0];
    for (int h = tid; h < 9 * NH; h += TX * TY) {
      const int c = h / NH, e = h - c * NH;
      int col, row;
      if (e < NHX) {
        row = e / (HXL + HXR);
        const int cx = e - row * (HXL + HXR);
        col = cx < HXL ? cx - HXL : TX + cx - HXL;
      } else {
        const int e2 = e - NHX;
        col = e2 % TX;
        const int ry = e2 / TX;
        row = ry < HYL ? ry - HYL : TY + ry - HYL;
      }
      const int Ih = blockIdx.x * TX + col + NG, Jh = blockIdx.y * TY + row + NG;
      float v = 0.f;
      if (Ih >= 0 && Ih < g.nx && Jh >= 0 && Jh < g.ny) v = __ldg(cur + c * sc + g.at(Ih, Jh, K));
      tile[c][row + HYL][col + HXL] = v;
    }
    __syncthreads();

    bool work = inside;
    if (work && slab_f >= 0 && (__ldg(a.fflag[slab_f] + J + (long)K * g.ny) & FL_SPLIT)) work = false;
    if (work) {
      float e[3][3];
#pragma unroll
      for (int qq = 0; qq < 9; qq++) e[qq / 3][qq % 3] = __ldg(a.met + (1 + qq) * sc + p);
      const float lam = __ldg(a.med + p), mu = __ldg(a.med + sc + p), slw = __ldg(a.med + 2 * sc + p);
      const float l2m = lam + 2.0f * mu;
      const bool top = a.isfree && K >= nk2 - 3;
      const bool surfrow = a.isfree && K == nk2;
      const long fidx = ((long)J * g.nx + I) * 9;
      float h[9], corr[9], r[9], D[9];
#pragma unroll
      for (int c = 0; c < 9; c++) corr[c] = 0.f;
      float dvx[3], dvy[3];
      // x
#pragma unroll
      for (int c = 0; c < 9; c++) {
        float s = 0.f;
#pragma unroll
        for (int n = 0; n < 5; n++) s += wdrp<ID>(n) * tile[c][ty + HYL][tx + HXL + (ID ? n - 1 : n - 3)];
        D[c] = s;
      }
      dvx[0] = D[VX]; dvx[1] = D[VY]; dvx[2] = D[VZ];
      rhs_dir(D, e[0], lam, mu, l2m, slw, r);
#pragma unroll
      for (int c = 0; c < 9; c++) h[c] = r[c];
      if (a.pml[0].on) pml_face<MODE>(a, a.pml[0], 0, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
      if (a.pml[1].on) pml_face<MODE>(a, a.pml[1], 0, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
      // y
#pragma unroll
      for (int c = 0; c < 9; c++) {
        float s = 0.f;
#pragma unroll
        for (int n = 0; n < 5; n++) s += wdrp<JD>(n) * tile[c][ty + HYL + (JD ? n - 1 : n - 3)][tx + HXL];
        D[c] = s;
      }
      dvy[0] = D[VX]; dvy[1] = D[VY]; dvy[2] = D[VZ];
      rhs_dir(D, e[1], lam, mu, l2m, slw, r);
#pragma unroll
      for (int c = 0; c < 9; c++) h[c] += r[c];
      if (a.pml[2].on) pml_face<MODE>(a, a.pml[2], 1, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
      if (a.pml[3].on) pml_face<MODE>(a, a.pml[3], 1, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
      // z
#pragma unroll
      for (int c = 0; c < 9; c++) {
        float s = 0.f;
#pragma unroll
        for (int n = 0; n < 5; n++) s += wdrp<KD>(n) * q[c][n];
        D[c] = s;
      }
      rhs_dir(D, e[2], lam, mu, l2m, slw, r);
      if (a.pml[4].on) pml_face<MODE>(a, a.pml[4], 2, I, J, K, r, D, e[2], lam, mu, l2m, false, fidx, corr);
      if (a.pml[5].on) pml_face<MODE>(a, a.pml[5], 2, I, J, K, r, D, e[2], lam, mu, l2m, false, fidx, corr);
      if (top && K >= nk2 - 2) {
        // velocity below the surface: the z part of the velocity gradient
        // comes from the conversion matrices (surface) or from 2nd / 4th
        // order one-sided differences (one / two rows below)
        float dz[3];
        if (K == nk2) {
          const float *X = a.free_mat + fidx;
          const float *Y = X + (long)g.ny * g.nx * 9;
          float o1[3], o2[3];
          mv3(X, dvx, o1); mv3(Y, dvy, o2);
          dz[0] = o1[0] + o2[0]; dz[1] = o1[1] + o2[1]; dz[2] = o1[2] + o2[2];
        } else if (K == nk2 - 1) {
#pragma unroll
          for (int c = 0; c < 3; c++) dz[c] = KD ? q[c][M0 + 1] - q[c][M0] : q[c][M0] - q[c][M0 - 1];
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++)
            dz[c] = KD ? kB1 * q[c][M0] + kB2 * q[c][M0 + 1] + kB3 * q[c][M0 + 2]
                       : -(kB1 * q[c][M0] + kB2 * q[c][M0 - 1] + kB3 * q[c][M0 - 2]);
        }
        float Dz[9];
#pragma unroll
        for (int c = 0; c < 9; c++) Dz[c] = 0.f;
        Dz[VX] = dz[0]; Dz[VY] = dz[1]; Dz[VZ] = dz[2];
        float rz[9];
        rhs_dir(Dz, e[2], lam, mu, l2m, slw, rz);
#pragma unroll
        for (int c = TXX; c <= TXY; c++) h[c] += rz[c];
#pragma unroll
        for (int c = VX; c <= VZ; c++) h[c] += r[c];
      } else {
#pragma unroll
        for (int c = 0; c < 9; c++) h[c] += r[c];
      }
      if (top && K >= nk2 - (KD ? 3 : 1)) {
        // traction image on the momentum equation in the top rows
        const float sj = slw / __ldg(a.met + MJAC * sc + p);
#pragma unroll 1
        for (int rr = 0; rr < 3; rr++) {
          float dx = 0.f, dy = 0.f, dzz = 0.f;
#pragma unroll
          for (int n = 0; n < 5; n++) dx += wdrp<ID>(n) * ctrac_t(cur, a.met, sc, p + (ID ? n - 1 : n - 3), MXIX, rr);
#pragma unroll
          for (int n = 0; n < 5; n++) dy += wdrp<JD>(n) * ctrac_t(cur, a.met, sc, p + (JD ? n - 1 : n - 3) * sy, METX, rr);
#pragma unroll
          for (int n = 0; n < 5; n++) {
            const int kk = K + (KD ? n - 1 : n - 3);
            float v = 0.f;
            if (kk < nk2) v = ctrac_t(cur, a.met, sc, g.at(I, J, kk), MZTX, rr);
            else if (kk > nk2) v = -ctrac_t(cur, a.met, sc, g.at(I, J, 2 * nk2 - kk), MZTX, rr);
            dzz += wdrp<KD>(n) * v;
          }
          h[VX + rr] = (dx + dy + dzz) * sj;
        }
      }
      // RK stage update
#pragma unroll
      for (int c = 0; c < 9; c++) {
        const long o = c * sc + p;
        const float hv = h[c] + corr[c];
        if (MODE == RK_FIRST) {
          const float v = q[c][M0];
          a.out[o] = v + a.ca * hv;
          a.end[o] = v + a.cb * hv;
        } else if (MODE == RK_MID) {
          a.out[o] = __ldg(a.pre + o) + a.ca * hv;
          a.end[o] += a.cb * hv;
        } else {
          a.end[o] += a.cb * hv;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 9; c++) {
#pragma unroll
      for (int m = 0; m < 4; m++) q[c][m] = q[c][m + 1];
    }
  }
}

template <int ID, int JD, int KD>
void launch_t(const VolArgs &a, int mode, cudaStream_t st) {
  const dim3 blk(TX, TY, 1);
  const dim3 grd((a.g.ni + TX - 1) / TX, (a.g.nj + TY - 1) / TY, (a.g.nk + a.kchunk - 1) / a.kchunk);
  if (mode == RK_FIRST) k_volume_tiled<ID, JD, KD, RK_FIRST><<<grd, blk, 0, st>>>(a);
  else if (mode == RK_MID) k_volume_tiled<ID, JD, KD, RK_MID><<<grd, blk, 0, st>>>(a);
  else k_volume_tiled<ID, JD, KD, RK_LAST><<<grd, blk, 0, st>>>(a);
}

}  // namespace

void launch_volume_tiled(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  switch (idir * 4 + jdir * 2 + kdir) {
    case 0: launch_t<0, 0, 0>(a, mode, st); break;
    case 1: launch_t<0, 0, 1>(a, mode, st); break;
    case 2: launch_t<0, 1, 0>(a, mode, st); break;
    case 3: launch_t<0, 1, 1>(a, mode, st); break;
    case 4: launch_t<1, 0, 0>(a, mode, st); break;
    case 5: launch_t<1, 0, 1>(a, mode, st); break;
    case 6: launch_t<1, 1, 0>(a, mode, st); break;
    default: launch_t<1, 1, 1>(a, mode, st); break;
  }
}

}  // namespace cgfd
