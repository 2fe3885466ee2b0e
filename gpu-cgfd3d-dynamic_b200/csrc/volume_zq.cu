// volume_zq.cu -- z-marching volume stage kernel for the interior box.
//
// Same arithmetic as the interior box kernel of volume.cu (inner stencil,
// sv_curv_col_el_iso_rhs_inner_gpu, src/forward/sv_curv_col_el_iso_gpu.cu:
// 232-388, and the RK stage update, wav_t.cu:219-234), laid out so that each
// wavefield value is fetched from HBM/L2 about once per stage:
//
//   * a block owns a 32 x 8 column of (x, y) points and marches up a chunk
//     of z rows;
//   * each thread keeps, per component, the five z samples the one-sided z
//     operator needs in registers; a step shifts the queue and adds the
//     leading plane, which was prefetched one step earlier;
//   * the current plane's nine components go to a double-buffered shared
//     memory tile with the one-sided x / y halo of this stage's operators
//     (1 point behind, 3 ahead, or the mirror), so x and y taps are shared
//     memory reads; the halo values are also prefetched one step ahead;
//   * one __syncthreads per z step (the double buffer makes the second
//     one unnecessary).
//
// Global traffic per point and stage: 9 leading-plane loads + ~5.6 halo
// loads (L2) + 12 coefficient loads + the RK level reads / writes, against
// ~129 loads of the box kernel, whose z taps always miss L1.
//
// Roofline: HBM-bound, 192 floats = 768 B per point and step (21+18,
// 39+18, 39+18, 30+9 floats over the 4 stages).
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

constexpr int ZX = 32, ZY = 8;
constexpr int SW = ZX + 4, SH = ZY + 4;   // tile with a 4-point halo per axis
constexpr int NHALO = 4 * ZY + 4 * ZX;    // halo points of one component
constexpr int NHT = (9 * NHALO + ZX * ZY - 1) / (ZX * ZY);   // halo loads per thread

// one-sided DRP derivative from shared memory; s points at the centre
template <int F>
__device__ __forceinline__ float dsm(const float *s, int st, float v0) {
  if (F) return kC1 * s[-st] + kC2 * v0 + kC3 * s[st] + kC4 * s[2 * st] + kC5 * s[3 * st];
  return -(kC5 * s[-3 * st] + kC4 * s[-2 * st] + kC3 * s[-st] + kC2 * v0 + kC1 * s[st]);
}

// one-sided DRP derivative from the z queue: planes k-1..k+3 (F) or
// k-3..k+1 (B)
template <int F>
__device__ __forceinline__ float dq(const float *q) {
  if (F) return kC1 * q[0] + kC2 * q[1] + kC3 * q[2] + kC4 * q[3] + kC5 * q[4];
  return -(kC5 * q[0] + kC4 * q[1] + kC3 * q[2] + kC2 * q[3] + kC1 * q[4]);
}

// halo slot t of the tile -> (component, tile row, tile column)
template <int XL, int YL>
__device__ __forceinline__ void halo_slot(int t, int &c, int &row, int &col) {
  c = t / NHALO;
  const int r = t - c * NHALO;
  if (r < 4 * ZX) {                 // y halo rows, full width
    const int hy = r / ZX;
    row = hy < YL ? hy : hy + ZY;
    col = XL + (r - hy * ZX);
  } else {                          // x halo columns, tile height
    const int r2 = r - 4 * ZX, hx = r2 / ZY;
    col = hx < XL ? hx : hx + ZX;
    row = YL + (r2 - hx * ZY);
  }
}

template <int ID, int JD, int KD, int MODE>
__global__ void __launch_bounds__(ZX * ZY, 2) k_interior_zq(const __grid_constant__ VolArgs a) {
  constexpr int XL = ID ? 1 : 3, YL = JD ? 1 : 3;      // halo behind the tile
  constexpr int LEAD = KD ? 3 : 1, BACK = KD ? 1 : 3;  // z reach ahead / behind
  __shared__ float sm[2][9][SH][SW];

  const Grid &g = a.g;
  const VolBox &B = a.box[0];
  const int bid = blockIdx.x;
  const int bx = bid % B.nbx, rem = bid / B.nbx, by = rem % B.nby, bz = rem / B.nby;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * ZX + tx;
  const int ti0 = B.i0 + bx * ZX, tj0 = B.j0 + by * ZY;    // tile origin (interior indices)
  const int i = ti0 + tx, j = tj0 + ty;
  const int kb = B.k0 + bz * a.kchunk;
  const int ke = min(kb + a.kchunk, a.kend);
  const bool act = i <= B.i1 && j <= B.j1;
  // points up to 3 beyond the box are read as taps; further ones are never
  // used and may lie outside the allocation
  const bool ld = i <= B.i1 + 3 && j <= B.j1 + 3;
  const long sc = g.scmp, sz = g.sz;
  const int I = i + NG, J = j + NG;
  const long pcol = g.at(I, J, 0);       // this column at K = 0

  // halo slots of this thread: tile slot (bit 20 set: outside the reach of
  // the taps, zero filled), component and in-plane offset
  int hslot[NHT], hc[NHT], hpl[NHT];
#pragma unroll
  for (int u = 0; u < NHT; u++) {
    const int t = tid + u * ZX * ZY;
    hslot[u] = -1;
    hc[u] = 0;
    hpl[u] = 0;
    if (t < 9 * NHALO) {
      int c, row, col;
      halo_slot<XL, YL>(t, c, row, col);
      const int hi = ti0 + col - XL, hj = tj0 + row - YL;
      hslot[u] = (c * SH + row) * SW + col;
      hc[u] = c;
      if (hi <= B.i1 + 3 && hj <= B.j1 + 3) hpl[u] = (int)g.at(hi + NG, hj + NG, 0);
      else hslot[u] |= 1 << 20;
    }
  }
  auto halo_ld = [&](int u, int K) {
    return (hslot[u] >= 0 && hslot[u] < (1 << 20)) ? __ldg(a.cur + (long)hc[u] * sc + hpl[u] + (long)K * sz) : 0.f;
  };

  // prime the queue with planes kb-BACK .. kb+LEAD-1; prefetch the leading
  // plane kb+LEAD and the halo of plane kb
  float q[9][5], nx[9], hv[NHT];
#pragma unroll
  for (int c = 0; c < 9; c++) {
#pragma unroll
    for (int l = 1; l < 5; l++) q[c][l] = ld ? __ldg(a.cur + c * sc + pcol + (long)(kb - BACK + l - 1 + NG) * sz) : 0.f;
    nx[c] = ld ? __ldg(a.cur + c * sc + pcol + (long)(kb + LEAD + NG) * sz) : 0.f;
  }
#pragma unroll
  for (int u = 0; u < NHT; u++) hv[u] = halo_ld(u, kb + NG);

  int buf = 0;
#pragma unroll 1
  for (int k = kb; k < ke; k++) {
    const int K = k + NG;
    // shift the queue: planes k-BACK .. k+LEAD
#pragma unroll
    for (int c = 0; c < 9; c++) {
#pragma unroll
      for (int l = 0; l < 4; l++) q[c][l] = q[c][l + 1];
      q[c][4] = nx[c];
    }
    float *S = &sm[buf][0][0][0];
#pragma unroll
    for (int c = 0; c < 9; c++) S[(c * SH + YL + ty) * SW + XL + tx] = q[c][BACK];
#pragma unroll
    for (int u = 0; u < NHT; u++)
      if (hslot[u] >= 0) S[hslot[u] & ((1 << 20) - 1)] = hv[u];
    __syncthreads();

    // prefetch plane k+1+LEAD and the halo of plane k+1
    if (k + 1 < ke) {
#pragma unroll
      for (int c = 0; c < 9; c++)
        nx[c] = ld ? __ldg(a.cur + c * sc + pcol + (long)(K + 1 + LEAD) * sz) : 0.f;
#pragma unroll
      for (int u = 0; u < NHT; u++) hv[u] = halo_ld(u, K + 1);
    }

    bool own = act;
    for (int f = 0; f < a.nfault; f++) {
      const int d = I - a.fi0[f];
      if (d >= -3 && d <= 3 && (__ldg(a.fflag[f] + J + (long)K * g.ny) & FL_SPLIT)) own = false;
    }
    if (own) {
      const long p = pcol + (long)K * sz;
      float e[3][3];
#pragma unroll
      for (int r = 0; r < 9; r++) e[r / 3][r % 3] = __ldg(a.met + (1 + r) * sc + p);
      const float lam = __ldg(a.med + p), mu = __ldg(a.med + sc + p), slw = __ldg(a.med + 2 * sc + p);
      float G[3][3], s[3];
      // x
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float d = dsm<ID>(S + (c * SH + YL + ty) * SW + XL + tx, 1, q[c][BACK]);
        G[c][0] = e[0][0] * d; G[c][1] = e[0][1] * d; G[c][2] = e[0][2] * d;
      }
      {
        const float *c0 = S + (YL + ty) * SW + XL + tx;
        float d;
        d = dsm<ID>(c0 + TXX * SH * SW, 1, q[TXX][BACK]); s[0] = e[0][0] * d;
        d = dsm<ID>(c0 + TYY * SH * SW, 1, q[TYY][BACK]); s[1] = e[0][1] * d;
        d = dsm<ID>(c0 + TZZ * SH * SW, 1, q[TZZ][BACK]); s[2] = e[0][2] * d;
        d = dsm<ID>(c0 + TYZ * SH * SW, 1, q[TYZ][BACK]); s[1] += e[0][2] * d; s[2] += e[0][1] * d;
        d = dsm<ID>(c0 + TXZ * SH * SW, 1, q[TXZ][BACK]); s[0] += e[0][2] * d; s[2] += e[0][0] * d;
        d = dsm<ID>(c0 + TXY * SH * SW, 1, q[TXY][BACK]); s[0] += e[0][1] * d; s[1] += e[0][0] * d;
      }
      // y
      {
        const float *c0 = S + (YL + ty) * SW + XL + tx;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float d = dsm<JD>(c0 + c * SH * SW, SW, q[c][BACK]);
          G[c][0] += e[1][0] * d; G[c][1] += e[1][1] * d; G[c][2] += e[1][2] * d;
        }
        float d;
        d = dsm<JD>(c0 + TXX * SH * SW, SW, q[TXX][BACK]); s[0] += e[1][0] * d;
        d = dsm<JD>(c0 + TYY * SH * SW, SW, q[TYY][BACK]); s[1] += e[1][1] * d;
        d = dsm<JD>(c0 + TZZ * SH * SW, SW, q[TZZ][BACK]); s[2] += e[1][2] * d;
        d = dsm<JD>(c0 + TYZ * SH * SW, SW, q[TYZ][BACK]); s[1] += e[1][2] * d; s[2] += e[1][1] * d;
        d = dsm<JD>(c0 + TXZ * SH * SW, SW, q[TXZ][BACK]); s[0] += e[1][2] * d; s[2] += e[1][0] * d;
        d = dsm<JD>(c0 + TXY * SH * SW, SW, q[TXY][BACK]); s[0] += e[1][1] * d; s[1] += e[1][0] * d;
      }
      // z
      {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float d = dq<KD>(q[c]);
          G[c][0] += e[2][0] * d; G[c][1] += e[2][1] * d; G[c][2] += e[2][2] * d;
        }
        float d;
        d = dq<KD>(q[TXX]); s[0] += e[2][0] * d;
        d = dq<KD>(q[TYY]); s[1] += e[2][1] * d;
        d = dq<KD>(q[TZZ]); s[2] += e[2][2] * d;
        d = dq<KD>(q[TYZ]); s[1] += e[2][2] * d; s[2] += e[2][1] * d;
        d = dq<KD>(q[TXZ]); s[0] += e[2][2] * d; s[2] += e[2][0] * d;
        d = dq<KD>(q[TXY]); s[0] += e[2][1] * d; s[1] += e[2][0] * d;
      }
      const float l2m = lam + 2.0f * mu;
      float h[9];
      h[VX] = slw * s[0]; h[VY] = slw * s[1]; h[VZ] = slw * s[2];
      h[TXX] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]);
      h[TYY] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]);
      h[TZZ] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]);
      h[TXY] = mu * (G[0][1] + G[1][0]);
      h[TXZ] = mu * (G[0][2] + G[2][0]);
      h[TYZ] = mu * (G[1][2] + G[2][1]);
      // RK update; level reads before the first store (the compiler cannot
      // prove that out and end do not alias)
      if (MODE == RK_FIRST) {
#pragma unroll
        for (int c = 0; c < 9; c++) {
          a.out[c * sc + p] = q[c][BACK] + a.ca * h[c];
          a.end[c * sc + p] = q[c][BACK] + a.cb * h[c];
        }
      } else {
        float pv[9], ev[9];
#pragma unroll
        for (int c = 0; c < 9; c++) {
          if (MODE == RK_MID) pv[c] = __ldg(a.pre + c * sc + p);
          ev[c] = a.end[c * sc + p];
        }
#pragma unroll
        for (int c = 0; c < 9; c++) {
          if (MODE == RK_MID) a.out[c * sc + p] = pv[c] + a.ca * h[c];
          a.end[c * sc + p] = ev[c] + a.cb * h[c];
        }
      }
    }
    buf ^= 1;
  }
}

template <int ID, int JD, int KD>
void launch_zq4(const VolArgs &a, int mode, cudaStream_t st) {
  const dim3 blk(ZX, ZY, 1), grd(a.nblocks);
  if (mode == RK_FIRST) k_interior_zq<ID, JD, KD, RK_FIRST><<<grd, blk, 0, st>>>(a);
  else if (mode == RK_MID) k_interior_zq<ID, JD, KD, RK_MID><<<grd, blk, 0, st>>>(a);
  else k_interior_zq<ID, JD, KD, RK_LAST><<<grd, blk, 0, st>>>(a);
}

}  // namespace

// block layout of the z-marching kernel over one box (interior indices,
// inclusive): tiles of 32 x 8 columns, chunks of kchunk rows
void volume_zq_layout(VolArgs &a, const int box[6], int kchunk) {
  a.nbox = 0;
  a.nblocks = 0;
  if (box[1] < box[0] || box[3] < box[2] || box[5] < box[4]) return;
  VolBox &B = a.box[0];
  B.i0 = box[0]; B.i1 = box[1]; B.j0 = box[2]; B.j1 = box[3]; B.k0 = box[4]; B.k1 = box[5];
  B.nbx = (box[1] - box[0] + ZX) / ZX;
  B.nby = (box[3] - box[2] + ZY) / ZY;
  B.first = 0;
  a.kchunk = kchunk;
  a.kend = box[5] + 1;
  const int nkc = (box[5] - box[4] + kchunk) / kchunk;
  a.nbox = 1;
  a.nblocks = B.nbx * B.nby * nkc;
}

void launch_volume_zq(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  if (a.nbox == 0) return;
  switch (idir * 4 + jdir * 2 + kdir) {
    case 0: launch_zq4<0, 0, 0>(a, mode, st); break;
    case 1: launch_zq4<0, 0, 1>(a, mode, st); break;
    case 2: launch_zq4<0, 1, 0>(a, mode, st); break;
    case 3: launch_zq4<0, 1, 1>(a, mode, st); break;
    case 4: launch_zq4<1, 0, 0>(a, mode, st); break;
    case 5: launch_zq4<1, 0, 1>(a, mode, st); break;
    case 6: launch_zq4<1, 1, 0>(a, mode, st); break;
    default: launch_zq4<1, 1, 1>(a, mode, st); break;
  }
}

}  // namespace cgfd
