// volume_sm.cu -- interior volume stage kernel with a shared-memory plane
// ring filled by cp.async.
//
// Same arithmetic as the interior box kernel of volume.cu (inner stencil,
// sv_curv_col_el_iso_rhs_inner_gpu, src/forward/sv_curv_col_el_iso_gpu.cu:
// 232-388, with the RK stage update of wav_t.cu:219-234), organised so that
// the stage input reaches the SM asynchronously, without registers:
//
//   * a block owns a 32 x 8 column of (x, y) points and marches up a chunk
//     of z rows;
//   * a ring of R = 5 + D planes in shared memory holds, per plane, the nine
//     components of the tile with a 4-point halo in x and y (1 behind and 3
//     ahead of the tile, or the mirror, for this stage's operators); the
//     five planes the z operator reaches are resident while the next are
//     in flight (cp.async, 4 bytes per thread and element, zero fill beyond
//     the reach of the taps);
//   * x, y and z taps are shared-memory reads; the metric, the medium and
//     the RK levels are read from global memory once per point;
//   * one __syncthreads per plane: the slot a plane is loaded into held the
//     plane read one iteration earlier.
//
// Roofline: HBM-bound, 192 floats = 768 B per point and step.
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

constexpr int SX = 32, SY = 8;                 // tile (threads)
constexpr int SW = SX + 4, SH = SY + 4;        // tile with halo
constexpr int PLANE = 9 * SH * SW;             // floats of one ring slot
constexpr int NHALO = SH * SW - SX * SY;       // halo points of one component (176)
constexpr int DEPTH = 2;                       // planes in flight ahead of the taps
constexpr int RING = 5 + DEPTH;
constexpr int SMEM_BYTES = RING * PLANE * 4;

__device__ __forceinline__ void cp_async4(unsigned dst, const float *src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int F>
__device__ __forceinline__ float dsm(const float *s, int st, float v0) {
  if (F) return kC1 * s[-st] + kC2 * v0 + kC3 * s[st] + kC4 * s[2 * st] + kC5 * s[3 * st];
  return -(kC5 * s[-3 * st] + kC4 * s[-2 * st] + kC3 * s[-st] + kC2 * v0 + kC1 * s[st]);
}

template <int ID, int JD, int KD, int MODE>
__global__ void __launch_bounds__(SX * SY, 2) k_interior_sm(const __grid_constant__ VolArgs a) {
  constexpr int XL = ID ? 1 : 3, YL = JD ? 1 : 3;      // halo behind the tile
  constexpr int LEAD = KD ? 3 : 1, BACK = KD ? 1 : 3;  // z reach ahead / behind
  extern __shared__ __align__(16) float ring[];

  const Grid &g = a.g;
  const VolBox &B = a.box[0];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SX + tx;
  const int ti0 = B.i0 + blockIdx.x * SX, tj0 = B.j0 + blockIdx.y * SY;   // tile origin
  const int i = ti0 + tx, j = tj0 + ty;
  const int kb = B.k0 + blockIdx.z * a.kchunk;
  const int ke = min(kb + a.kchunk, a.kend);
  const bool act = i <= B.i1 && j <= B.j1;
  const long sc = g.scmp, sz = g.sz;
  const int I = i + NG, J = j + NG;
  const long pcol = g.at(I, J, 0);

  // what this thread copies into a ring slot: its own point and (tid < 176)
  // one halo point, for each component; points more than 3 beyond the box
  // are never read by a tap and may lie outside the allocation (zero fill)
  const bool own_ok = i <= B.i1 + 3 && j <= B.j1 + 3;
  const int own_s = (YL + ty) * SW + XL + tx;
  int halo_s = 0;
  long halo_g = 0;
  bool halo_ok = false;
  const bool has_halo = tid < NHALO;
  if (has_halo) {
    int row, col;
    if (tid < 4 * SW) {
      const int hr = tid / SW;
      row = hr < YL ? hr : hr + SY;
      col = tid - hr * SW;
    } else {
      const int h2 = tid - 4 * SW, hc = h2 & 3;
      row = YL + (h2 >> 2);
      col = hc < XL ? hc : hc + SX;
    }
    const int hi = ti0 + col - XL, hj = tj0 + row - YL;
    halo_s = row * SW + col;
    halo_ok = hi <= B.i1 + 3 && hj <= B.j1 + 3;
    halo_g = halo_ok ? g.at(hi + NG, hj + NG, 0) : pcol;
  }
  const unsigned ring_s = static_cast<unsigned>(__cvta_generic_to_shared(ring));
  auto load_plane = [&](int K) {
    const unsigned base = ring_s + (unsigned)((K % RING) * PLANE) * 4u;
    const long zo = (long)K * sz;
#pragma unroll
    for (int c = 0; c < 9; c++) {
      const float *src = a.cur + c * sc + zo;
      cp_async4(base + (unsigned)(c * SH * SW + own_s) * 4u, src + (own_ok ? pcol : 0), own_ok);
      if (has_halo) cp_async4(base + (unsigned)(c * SH * SW + halo_s) * 4u, src + halo_g, halo_ok);
    }
    cp_commit();
  };

  // prologue: planes kb-BACK .. kb+LEAD+DEPTH-1, one commit group each
  const int Kb = kb + NG, Ke = ke + NG;
#pragma unroll 1
  for (int K = Kb - BACK; K < Kb + LEAD + DEPTH; K++) {
    if (K < Ke + LEAD) load_plane(K);
    else cp_commit();
  }

#pragma unroll 1
  for (int K = Kb; K < Ke; K++) {
    // one group per plane, in plane order; the newest issued is plane
    // K+LEAD+DEPTH-1, so with all but the DEPTH-1 newest complete, plane
    // K+LEAD (the farthest tap) is in
    cp_wait<DEPTH - 1>();
    __syncthreads();
    // refill the slot of plane K-BACK-1 (read in the previous iteration)
    if (K + LEAD + DEPTH < Ke + LEAD) load_plane(K + LEAD + DEPTH);
    else cp_commit();

    bool own = act;
    for (int f = 0; f < a.nfault; f++) {
      const int d = I - a.fi0[f];
      if (d >= -3 && d <= 3 && (__ldg(a.fflag[f] + J + (long)K * g.ny) & FL_SPLIT)) own = false;
    }
    if (!own) continue;
    const long p = pcol + (long)K * sz;
    float e[3][3];
#pragma unroll
    for (int r = 0; r < 9; r++) e[r / 3][r % 3] = __ldg(a.met + (1 + r) * sc + p);
    const float lam = __ldg(a.med + p), mu = __ldg(a.med + sc + p), slw = __ldg(a.med + 2 * sc + p);

    const float *S = ring + (K % RING) * PLANE + own_s;   // this point, component 0, plane K
    float v0[9];
#pragma unroll
    for (int c = 0; c < 9; c++) v0[c] = S[c * SH * SW];
    // z taps: the same point in the ring slots of planes K-1..K+3 (F) or K-3..K+1 (B)
    auto zs = [&](int dk) { return ring + ((K + dk) % RING) * PLANE + own_s; };
    const float *z0 = KD ? zs(-1) : zs(-3);
    const float *z1 = KD ? zs(1) : zs(-2);
    const float *z2 = KD ? zs(2) : zs(-1);
    const float *z3 = KD ? zs(3) : zs(1);
    auto dz = [&](int c) {
      const int o = c * SH * SW;
      if (KD) return kC1 * z0[o] + kC2 * v0[c] + kC3 * z1[o] + kC4 * z2[o] + kC5 * z3[o];
      return -(kC5 * z0[o] + kC4 * z1[o] + kC3 * z2[o] + kC2 * v0[c] + kC1 * z3[o]);
    };

    float G[3][3], s[3];
    // x
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float d = dsm<ID>(S + c * SH * SW, 1, v0[c]);
      G[c][0] = e[0][0] * d; G[c][1] = e[0][1] * d; G[c][2] = e[0][2] * d;
    }
    {
      float d;
      d = dsm<ID>(S + TXX * SH * SW, 1, v0[TXX]); s[0] = e[0][0] * d;
      d = dsm<ID>(S + TYY * SH * SW, 1, v0[TYY]); s[1] = e[0][1] * d;
      d = dsm<ID>(S + TZZ * SH * SW, 1, v0[TZZ]); s[2] = e[0][2] * d;
      d = dsm<ID>(S + TYZ * SH * SW, 1, v0[TYZ]); s[1] += e[0][2] * d; s[2] += e[0][1] * d;
      d = dsm<ID>(S + TXZ * SH * SW, 1, v0[TXZ]); s[0] += e[0][2] * d; s[2] += e[0][0] * d;
      d = dsm<ID>(S + TXY * SH * SW, 1, v0[TXY]); s[0] += e[0][1] * d; s[1] += e[0][0] * d;
    }
    // y
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float d = dsm<JD>(S + c * SH * SW, SW, v0[c]);
      G[c][0] += e[1][0] * d; G[c][1] += e[1][1] * d; G[c][2] += e[1][2] * d;
    }
    {
      float d;
      d = dsm<JD>(S + TXX * SH * SW, SW, v0[TXX]); s[0] += e[1][0] * d;
      d = dsm<JD>(S + TYY * SH * SW, SW, v0[TYY]); s[1] += e[1][1] * d;
      d = dsm<JD>(S + TZZ * SH * SW, SW, v0[TZZ]); s[2] += e[1][2] * d;
      d = dsm<JD>(S + TYZ * SH * SW, SW, v0[TYZ]); s[1] += e[1][2] * d; s[2] += e[1][1] * d;
      d = dsm<JD>(S + TXZ * SH * SW, SW, v0[TXZ]); s[0] += e[1][2] * d; s[2] += e[1][0] * d;
      d = dsm<JD>(S + TXY * SH * SW, SW, v0[TXY]); s[0] += e[1][1] * d; s[1] += e[1][0] * d;
    }
    // z
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float d = dz(c);
      G[c][0] += e[2][0] * d; G[c][1] += e[2][1] * d; G[c][2] += e[2][2] * d;
    }
    {
      float d;
      d = dz(TXX); s[0] += e[2][0] * d;
      d = dz(TYY); s[1] += e[2][1] * d;
      d = dz(TZZ); s[2] += e[2][2] * d;
      d = dz(TYZ); s[1] += e[2][2] * d; s[2] += e[2][1] * d;
      d = dz(TXZ); s[0] += e[2][2] * d; s[2] += e[2][0] * d;
      d = dz(TXY); s[0] += e[2][1] * d; s[1] += e[2][0] * d;
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
        a.out[c * sc + p] = v0[c] + a.ca * h[c];
        a.end[c * sc + p] = v0[c] + a.cb * h[c];
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
  // no copy may be in flight when the block exits
  cp_wait<0>();
}

template <int ID, int JD, int KD>
void launch_sm4(const VolArgs &a, int mode, cudaStream_t st) {
  const VolBox &B = a.box[0];
  const int nkc = (a.kend - B.k0 + a.kchunk - 1) / a.kchunk;
  const dim3 blk(SX, SY, 1), grd(B.nbx, B.nby, nkc);
  if (mode == RK_FIRST) k_interior_sm<ID, JD, KD, RK_FIRST><<<grd, blk, SMEM_BYTES, st>>>(a);
  else if (mode == RK_MID) k_interior_sm<ID, JD, KD, RK_MID><<<grd, blk, SMEM_BYTES, st>>>(a);
  else k_interior_sm<ID, JD, KD, RK_LAST><<<grd, blk, SMEM_BYTES, st>>>(a);
}

template <int ID, int JD, int KD>
cudaError_t attr_sm4() {
  cudaError_t e = cudaSuccess;
  for (cudaError_t r : { cudaFuncSetAttribute(k_interior_sm<ID, JD, KD, RK_FIRST>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES),
                         cudaFuncSetAttribute(k_interior_sm<ID, JD, KD, RK_MID>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES),
                         cudaFuncSetAttribute(k_interior_sm<ID, JD, KD, RK_LAST>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) })
    if (r != cudaSuccess) e = r;
  return e;
}

}  // namespace

// allow the ring's dynamic shared memory for every instantiation; call once
// per device before the first launch (outside stream capture)
cudaError_t volume_sm_prepare() {
  cudaError_t e = cudaSuccess;
  for (cudaError_t r : { attr_sm4<0, 0, 0>(), attr_sm4<0, 0, 1>(), attr_sm4<0, 1, 0>(), attr_sm4<0, 1, 1>(),
                         attr_sm4<1, 0, 0>(), attr_sm4<1, 0, 1>(), attr_sm4<1, 1, 0>(), attr_sm4<1, 1, 1>() })
    if (r != cudaSuccess) e = r;
  return e;
}

// block layout over the interior box (interior indices, inclusive): 32 x 8
// tiles, chunks of kchunk z rows
void volume_sm_layout(VolArgs &a, const int box[6], int kchunk) {
  a.nbox = 0;
  a.nblocks = 0;
  if (box[1] < box[0] || box[3] < box[2] || box[5] < box[4]) return;
  VolBox &B = a.box[0];
  B.i0 = box[0]; B.i1 = box[1]; B.j0 = box[2]; B.j1 = box[3]; B.k0 = box[4]; B.k1 = box[5];
  B.nbx = (box[1] - box[0] + SX) / SX;
  B.nby = (box[3] - box[2] + SY) / SY;
  B.first = 0;
  a.kchunk = kchunk;
  a.kend = box[5] + 1;
  a.nbox = 1;
  a.nblocks = B.nbx * B.nby * ((box[5] - box[4] + kchunk) / kchunk);
}

void launch_volume_sm(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  if (a.nbox == 0) return;
  switch (idir * 4 + jdir * 2 + kdir) {
    case 0: launch_sm4<0, 0, 0>(a, mode, st); break;
    case 1: launch_sm4<0, 0, 1>(a, mode, st); break;
    case 2: launch_sm4<0, 1, 0>(a, mode, st); break;
    case 3: launch_sm4<0, 1, 1>(a, mode, st); break;
    case 4: launch_sm4<1, 0, 0>(a, mode, st); break;
    case 5: launch_sm4<1, 0, 1>(a, mode, st); break;
    case 6: launch_sm4<1, 1, 0>(a, mode, st); break;
    default: launch_sm4<1, 1, 1>(a, mode, st); break;
  }
}

}  // namespace cgfd
