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
// k_volume<INTERIOR>, whose code holds no boundary logic; slabs that one
// direction's PML faces reach run k_volume<FACE_X/Y/Z>; PML edges, corners
// and the bottom ring run k_volume<EDGE>; the four rows under the free
// surface run k_volume<TOP> away from the PML columns and k_volume<SHELL>
// in them; the fault planes' welded points next to split nodes run
// k_volume<PLANE> after the first fault kernels.  Each stage reads the
// input level (stencil taps come from L1/L2), the metric and the medium
// once and writes the output levels once; each thread asks L2 early for
// the lines it reads last (prefetch), and interior threads for the next z
// row's DRAM misses.
//
// A level stores the nine components of a point in two 16-byte groups and
// one real (Grid::w), so a stencil tap is three loads: x taps are
// immediate offsets from three base pointers, y / z taps share two int
// offset tables, the centre sample is loaded once for all three
// directions.  The RHS is built direction by direction, so a PML face of
// normal d reuses direction d's contribution.
//
// Roofline: HBM-bound.  Algorithmic traffic per point and step is
// 192 floats = 768 B (21+18, 39+18, 39+18, 30+9 floats over the 4 stages).
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

constexpr int BX = 32, BY = 8;


// conservative traction J * (e . sigma_row) at point q for metric row d
// (0: xi, 1: eta, 2: zeta), all three stress rows (xx,xy,xz), (xy,yy,yz),
// (xz,yz,zz)
__device__ __forceinline__ void ctrac3(const Grid &g, const real *__restrict__ w, const real *__restrict__ cf,
                                       long q, int d, real t[3]) {
  const real4 e = coef_row(cf, g.scmp, d, q);
  const real J = coef_jac(cf, q);
  const real sxx = __ldg(w + g.w(TXX, q)), sxy = __ldg(w + g.w(TXY, q));
  const real4 s4 = __ldg(reinterpret_cast<const real4 *>(w + 4 * g.scmp) + q);   // Tyy Tzz Tyz Txz
  const real syy = s4.x, szz = s4.y, syz = s4.z, sxz = s4.w;
  t[0] = J * (e.x * sxx + e.y * sxy + e.z * sxz);
  t[1] = J * (e.x * sxy + e.y * syy + e.z * syz);
  t[2] = J * (e.x * sxz + e.y * syz + e.z * szz);
}

// the point's three groups within one level
struct Taps {
  const real4 *__restrict__ a;  // Vx Vy Vz Txx
  const real4 *__restrict__ b;  // Tyy Tzz Tyz Txz
  const real *__restrict__ t;   // Txy
};
__device__ __forceinline__ Taps taps_at(const real *w, long sc, long p) {
  Taps T;
  T.a = reinterpret_cast<const real4 *>(w) + p;
  T.b = reinterpret_cast<const real4 *>(w + 4 * sc) + p;
  T.t = w + 8 * sc + p;
  return T;
}
// the nine components of the point o points away
__device__ __forceinline__ void ld9(const Taps &T, int o, real v[9]) {
  const real4 x = __ldg(T.a + o), y = __ldg(T.b + o);
  v[VX] = x.x; v[VY] = x.y; v[VZ] = x.z; v[TXX] = x.w;
  v[TYY] = y.x; v[TZZ] = y.y; v[TYZ] = y.z; v[TXZ] = y.w;
  v[TXY] = __ldg(T.t + o);
}

template <int F>
__device__ __forceinline__ real wdrp(int n) {
  return F ? (n == 0 ? kC1 : n == 1 ? kC2 : n == 2 ? kC3 : n == 3 ? kC4 : kC5)
           : (n == 0 ? -kC5 : n == 1 ? -kC4 : n == 2 ? -kC3 : n == 3 ? -kC2 : -kC1);
}

template <int F>
__device__ __forceinline__ void tap_offsets(int s, int off[4]) {
  if (F) { off[0] = -s; off[1] = s; off[2] = 2 * s; off[3] = 3 * s; }
  else { off[0] = -3 * s; off[1] = -2 * s; off[2] = -s; off[3] = s; }
}

// direction-d part of the RHS from the nine d-derivatives D[c] and e = e_d
__device__ __forceinline__ void rhs_dir(const real D[9], const real e[3], real lam, real mu, real l2m,
                                        real slw, real r[9]) {
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

// one-sided DRP derivatives of the nine components, the centre sample v0
// known; off[n] are the offsets of the 4 other taps in table order
// (F: -1, 0, 1, 2, 3; B: -3, -2, -1, 0, 1 with the centre at n = 1 / 3).
// Each tap's nine components come in one go; the sums keep the order of
// the coefficient table.
template <int F>
__device__ __forceinline__ void derivs(const Taps &T, const real v0[9], const int off[4], real D[9]) {
  real t[9];
  ld9(T, off[0], t);
#pragma unroll
  for (int c = 0; c < 9; c++) D[c] = (F ? kC1 : kC5) * t[c];
  if (F) {
#pragma unroll
    for (int c = 0; c < 9; c++) D[c] += kC2 * v0[c];
  }
  ld9(T, off[1], t);
#pragma unroll
  for (int c = 0; c < 9; c++) D[c] += (F ? kC3 : kC4) * t[c];
  ld9(T, off[2], t);
#pragma unroll
  for (int c = 0; c < 9; c++) D[c] += (F ? kC4 : kC3) * t[c];
  if (!F) {
#pragma unroll
    for (int c = 0; c < 9; c++) D[c] += kC2 * v0[c];
  }
  ld9(T, off[3], t);
#pragma unroll
  for (int c = 0; c < 9; c++) D[c] = F ? D[c] + kC5 * t[c] : -(D[c] + kC1 * t[c]);
}

// Accumulate one direction's derivatives straight into the velocity
// gradient G[c][b] = dV_c/dx_b and the momentum sums
// s_r = sum_a e_a . d(sigma_row r)/dxi_a.
template <int F>
__device__ __forceinline__ void acc_dir(const Taps &T, const real v0[9], const int off[4], const real ea[3],
                                        real G[3][3], real s[3]) {
  real D[9];
  derivs<F>(T, v0, off, D);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const real d = D[VX + c];
    G[c][0] += ea[0] * d; G[c][1] += ea[1] * d; G[c][2] += ea[2] * d;
  }
  s[0] += ea[0] * D[TXX];
  s[1] += ea[1] * D[TYY];
  s[2] += ea[2] * D[TZZ];
  s[1] += ea[2] * D[TYZ]; s[2] += ea[1] * D[TYZ];
  s[0] += ea[2] * D[TXZ]; s[2] += ea[0] * D[TXZ];
  s[0] += ea[1] * D[TXY]; s[1] += ea[0] * D[TXY];
}

// the nine components of point p of a level in the grouped layout with
// sc points per component (read-only data through the non-coherent path)
__device__ __forceinline__ void ld9(const real *w, long sc, long p, real v[9], bool ro) {
  const real4 *A = reinterpret_cast<const real4 *>(w) + p, *B = reinterpret_cast<const real4 *>(w + 4 * sc) + p;
  const real4 x = ro ? __ldg(A) : *A, y = ro ? __ldg(B) : *B;
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
  v[8] = ro ? __ldg(w + 8 * sc + p) : w[8 * sc + p];
}
// level value + k * h at point p of level w
__device__ __forceinline__ void st9(real *w, long sc, long p, const real v[9], real k, const real h[9]) {
  reinterpret_cast<real4 *>(w)[p] = make_real4(v[0] + k * h[0], v[1] + k * h[1], v[2] + k * h[2], v[3] + k * h[3]);
  reinterpret_cast<real4 *>(w + 4 * sc)[p] =
      make_real4(v[4] + k * h[4], v[5] + k * h[5], v[6] + k * h[6], v[7] + k * h[7]);
  w[8 * sc + p] = v[8] + k * h[8];
}
// L2 prefetch of the auxiliary-field lines that pml_face reads at (I, J, K)
template <int MODE>
__device__ __forceinline__ void pml_prefetch(const PmlFaceDev &P, int I, int J, int K) {
  const int li = I - P.i1, lj = J - P.j1, lk = K - P.k1;
  if (li < 0 || li >= P.fni || lj < 0 || lj >= P.fnj || lk < 0 || lk >= P.fnk) return;
  const long pa = li + (long)lj * P.fni + (long)lk * P.fni * P.fnj, sz = P.siz;
  const real *lv[3] = { P.acur, MODE == RK_MID ? P.apre : nullptr, MODE != RK_FIRST ? P.aend : nullptr };
#pragma unroll
  for (int l = 0; l < 3; l++) {
    if (!lv[l]) continue;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(lv[l] + 4 * pa));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(lv[l] + 4 * sz + 4 * pa));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(lv[l] + 8 * sz + pa));
  }
}

// PML face P (normal d) at this point: add its correction to corr and
// advance its auxiliary fields (stored like a wavefield level, grouped,
// with P.siz points per component)
template <int MODE>
__device__ __forceinline__ void pml_face(const VolArgs &a, const PmlFaceDev &P, int d, int I, int J, int K,
                                         const real r[9], const real D[9], const real e2[3], real lam,
                                         real mu, real l2m, bool surf, long fidx, real corr[9]) {
  const int li = I - P.i1, lj = J - P.j1, lk = K - P.k1;
  if (li < 0 || li >= P.fni || lj < 0 || lj >= P.fnj || lk < 0 || lk >= P.fnk) return;
  const int layer = d == 0 ? li : (d == 1 ? lj : lk);
  const real cA = __ldg(P.A + layer), cB = __ldg(P.B + layer), cD = __ldg(P.D + layer);
  const long pa = li + (long)lj * P.fni + (long)lk * P.fni * P.fnj;
  real ac[9], ar[9];
  ld9(P.acur, P.siz, pa, ac, true);
#pragma unroll
  for (int c = 0; c < 9; c++) {
    corr[c] += (cB - 1.0f) * r[c] - cB * ac[c];
    ar[c] = cD * r[c] - cA * ac[c];
  }
  if (surf) {
    // free-surface coupling of the x / y faces: the d-derivative of the
    // surface-converted dz velocity gradient
    const real *X = a.free_mat + (long)(d == 0 ? 0 : 1) * a.g.ny * a.g.nx * 9 + fidx;
    const real dd[3] = { D[VX], D[VY], D[VZ] };
    real z[3];
    mv3(X, dd, z);
    real q[9];
    q[TXX] = l2m * (e2[0] * z[0]) + lam * (e2[1] * z[1] + e2[2] * z[2]);
    q[TYY] = l2m * (e2[1] * z[1]) + lam * (e2[0] * z[0] + e2[2] * z[2]);
    q[TZZ] = l2m * (e2[2] * z[2]) + lam * (e2[0] * z[0] + e2[1] * z[1]);
    q[TXY] = mu * (e2[1] * z[0] + e2[0] * z[1]);
    q[TXZ] = mu * (e2[2] * z[0] + e2[0] * z[2]);
    q[TYZ] = mu * (e2[2] * z[1] + e2[1] * z[2]);
#pragma unroll
    for (int c = TXX; c <= TXY; c++) { corr[c] += (cB - 1.0f) * q[c]; ar[c] += cD * q[c]; }
  }
  // auxiliary RK update; level reads first (see rk_update)
  if (MODE == RK_FIRST) {
    st9(P.aout, P.siz, pa, ac, a.ca, ar);
    st9(P.aend, P.siz, pa, ac, a.cb, ar);
  } else {
    real pv[9], ev[9];
    if (MODE == RK_MID) ld9(P.apre, P.siz, pa, pv, true);
    ld9(P.aend, P.siz, pa, ev, false);
    if (MODE == RK_MID) st9(P.aout, P.siz, pa, pv, a.ca, ar);
    st9(P.aend, P.siz, pa, ev, a.cb, ar);
  }
}

// RK stage update of the nine components at p.  All reads of the levels
// are issued before the first store: the compiler cannot prove that out
// and end do not alias, and interleaved load / store pairs would cost one
// memory round trip per component.
template <int MODE>
__device__ __forceinline__ void rk_update(const VolArgs &a, long p, const real v0[9], const real h[9]) {
  const long sc = a.g.scmp;
  if (MODE == RK_FIRST) {
    st9(a.out, sc, p, v0, a.ca, h);
    st9(a.end, sc, p, v0, a.cb, h);
  } else {
    real pv[9], ev[9];
    if (MODE == RK_MID) ld9(a.pre, sc, p, pv, true);
    ld9(a.end, sc, p, ev, false);
    if (MODE == RK_MID) st9(a.out, sc, p, pv, a.ca, h);
    st9(a.end, sc, p, ev, a.cb, h);
  }
}

// kernel kinds: the interior box (no boundary logic), slabs that only PML
// faces of one direction reach (x, y or z), the generic shell (the rows
// under the free surface, with any PML faces), and the PML edges and
// corners away from the free surface (the shell's code without the
// free-surface logic, which keeps it in registers)
enum { INTERIOR = 0, SHELL = 1, FACE_X = 2, FACE_Y = 3, FACE_Z = 4, EDGE = 5, PLANE = 6, TOP = 7 };
// PLANE: the interior kernel's code on packed boxes: the fault planes
// x = i0 inside the interior box, when the interior launch defers them.
// TOP: the shell's code without the PML faces, for the rows under the free
// surface away from every PML face (fewer live values than the shell)

// block -> point; boxes with a narrow x extent (PML x slabs) pack their
// points densely instead of leaving most of a 32-wide row idle
__device__ __forceinline__ bool locate(const VolArgs &a, int &i, int &j, int &k) {
  int b = 0;
#pragma unroll 1
  while (b + 1 < a.nbox && (int)blockIdx.x >= a.box[b + 1].first) b++;
  const VolBox &B = a.box[b];
  const int bid = blockIdx.x - B.first;
  const int ni = B.i1 - B.i0 + 1, nj = B.j1 - B.j0 + 1;
  if (B.nbx == 0) {
    // packed: flat index over the (x, y) rectangle of one z row
    const int t = (bid % B.nby) * (BX * BY) + threadIdx.y * BX + threadIdx.x;
    k = B.k0 + bid / B.nby;
    if (t >= ni * nj) return false;
    i = B.i0 + t % ni;
    j = B.j0 + t / ni;
    return true;
  }
  const int bx = bid % B.nbx, rem = bid / B.nbx, by = rem % B.nby, bz = rem / B.nby;
  i = B.i0 + bx * BX + threadIdx.x;
  j = B.j0 + by * BY + threadIdx.y;
  k = B.k0 + bz;
  return i <= B.i1 && j <= B.j1;
}

// interior box (one box): 3-D grid (x tiles, y tiles of one chunk, z rows x
// chunks).  The blocks of one y chunk of a.ychunk tiles march up z before
// the next chunk starts, so the planes a z window touches stay in L2 (a
// whole xy plane per z row would need more than the 126 MB L2 holds).
__device__ __forceinline__ bool locate_interior(const VolArgs &a, int &i, int &j, int &k) {
  const VolBox &B = a.box[0];
  const int nkb = B.k1 - B.k0 + 1;
  const int chunk = blockIdx.z / nkb, bz = blockIdx.z - chunk * nkb;
  const int by = chunk * a.ychunk + blockIdx.y;
  i = B.i0 + blockIdx.x * BX + threadIdx.x;
  j = B.j0 + by * BY + threadIdx.y;
  k = B.k0 + bz;
  return i <= B.i1 && j <= B.j1;
}

#ifndef CGFD_PREFETCH
#define CGFD_PREFETCH 1
#endif
// interior kernel: z rows ahead whose DRAM misses each thread prefetches
// (0: none)
#ifndef CGFD_AHEAD
#define CGFD_AHEAD 1
#endif

// resident blocks per SM asked of the compiler, per kernel kind (register
// budget 65536 / (256 x blocks))
#ifndef CGFD_LB_INTERIOR
#define CGFD_LB_INTERIOR 4
#endif
#ifndef CGFD_LB_TOP
#define CGFD_LB_TOP 3
#endif
#ifndef CGFD_LB_SHELL
#define CGFD_LB_SHELL 3
#endif
#ifndef CGFD_LB_FACE
#define CGFD_LB_FACE 3
#endif

template <int ID, int JD, int KD, int MODE, int KIND>
__global__ void __launch_bounds__(BX * BY, KIND == INTERIOR || KIND == PLANE ? CGFD_LB_INTERIOR
                                         : (KIND == SHELL || KIND == EDGE ? CGFD_LB_SHELL
                                                                          : (KIND == TOP ? CGFD_LB_TOP : CGFD_LB_FACE)))
    k_volume(const __grid_constant__ VolArgs a) {
  static_assert(KIND >= INTERIOR && KIND <= TOP, "kernel kind");
  const Grid &g = a.g;
  int i, j, k;
  if (KIND == INTERIOR ? !locate_interior(a, i, j, k) : !locate(a, i, j, k)) return;
  const int I = i + NG, J = j + NG, K = k + NG;
  // split-node slabs (i0-3..i0+3 of unwelded nodes) belong to the fault
  // kernels; with defer_i0 the fault planes go to the PLANE launch
  for (int f = 0; f < a.nfault; f++) {
    const int d = I - a.fi0[f];
    if (KIND == INTERIOR && d == 0 && a.defer_i0 && J >= a.fdef[f][0] && J <= a.fdef[f][1] && K >= a.fdef[f][2] &&
        K <= a.fdef[f][3])
      return;
    if (d >= -3 && d <= 3 && (__ldg(a.fflag[f] + J + (long)K * g.ny) & FL_SPLIT)) return;
  }
  const long p = g.at(I, J, K);
  const long sc = g.scmp;
#if CGFD_PREFETCH
  if (MODE != RK_FIRST) {
    // the RK update reads the time-n level and the accumulator last: ask
    // L2 for their lines now, so that those reads wait on L2, not DRAM
    const real *q[6] = { a.end + 4 * p, a.end + 4 * sc + 4 * p, a.end + 8 * sc + p,
                          a.pre + 4 * p, a.pre + 4 * sc + 4 * p, a.pre + 8 * sc + p };
#pragma unroll
    for (int n = 0; n < (MODE == RK_MID ? 6 : 3); n++) asm volatile("prefetch.global.L2 [%0];" ::"l"(q[n]));
  }
#if CGFD_AHEAD > 0
  if (KIND == INTERIOR) {
    // the DRAM misses of the block CGFD_AHEAD z rows up: the newest stencil
    // plane of the stage input and its coefficients (that block runs soon
    // after this one: blocks march up z within a y chunk)
    const int kn = K + CGFD_AHEAD + (KD ? 3 : 1), kc = K + CGFD_AHEAD;
    if (kn < g.nz) {
      const long q = p + (long)(kn - K) * g.sz;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a.cur + 4 * q));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a.cur + 4 * sc + 4 * q));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a.cur + 8 * sc + q));
    }
    if (kc < g.nz) {
      const long q = p + (long)CGFD_AHEAD * g.sz;
#pragma unroll
      for (int d = 0; d < 3; d++) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.coef + sc + 4 * (d * sc + q)));
    }
  }
#endif
  // likewise the auxiliary fields of the PML faces this point lies in
  if (KIND != INTERIOR && KIND != PLANE && KIND != TOP) {
#pragma unroll
    for (int f = 0; f < 6; f++) {
      if (KIND >= FACE_X && KIND <= FACE_Z && f / 2 != KIND - FACE_X) continue;
      if (a.pml[f].on) pml_prefetch<MODE>(a.pml[f], I, J, K);
    }
  }
#endif
  const Taps w = taps_at(a.cur, sc, p);
  real v0[9];
  ld9(w, 0, v0);
  const real4 r0 = coef_row(a.coef, sc, 0, p), r1 = coef_row(a.coef, sc, 1, p), r2 = coef_row(a.coef, sc, 2, p);
  const real e[3][3] = { { r0.x, r0.y, r0.z }, { r1.x, r1.y, r1.z }, { r2.x, r2.y, r2.z } };
  const real lam = r0.w, mu = r1.w, slw = r2.w;
  const real l2m = lam + 2.0f * mu;
  int ox[4], oy[4], oz[4];
  tap_offsets<ID>(1, ox);
  tap_offsets<JD>((int)g.sy, oy);
  tap_offsets<KD>((int)g.sz, oz);

  real h[9];
  if (KIND == INTERIOR || KIND == PLANE) {
    real G[3][3] = { { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f } };
    real s[3] = { 0.f, 0.f, 0.f };
    acc_dir<ID>(w, v0, ox, e[0], G, s);
    acc_dir<JD>(w, v0, oy, e[1], G, s);
    acc_dir<KD>(w, v0, oz, e[2], G, s);
    h[VX] = slw * s[0]; h[VY] = slw * s[1]; h[VZ] = slw * s[2];
    h[TXX] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]);
    h[TYY] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]);
    h[TZZ] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]);
    h[TXY] = mu * (G[0][1] + G[1][0]);
    h[TXZ] = mu * (G[0][2] + G[2][0]);
    h[TYZ] = mu * (G[1][2] + G[2][1]);
    rk_update<MODE>(a, p, v0, h);
    return;
  }

  if constexpr (KIND >= FACE_X && KIND <= FACE_Z) {
    // one PML direction FD: the other two directions accumulate like the
    // interior, direction FD is kept apart for the face's correction and
    // auxiliary update
    constexpr int FD = KIND - FACE_X;
    constexpr int FF = FD == 0 ? ID : (FD == 1 ? JD : KD);
    real G[3][3] = { { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f } };
    real s[3] = { 0.f, 0.f, 0.f };
    if (FD != 0) acc_dir<ID>(w, v0, ox, e[0], G, s);
    if (FD != 1) acc_dir<JD>(w, v0, oy, e[1], G, s);
    if (FD != 2) acc_dir<KD>(w, v0, oz, e[2], G, s);
    real D[9], r[9], corr[9];
    derivs<FF>(w, v0, FD == 0 ? ox : (FD == 1 ? oy : oz), D);
    rhs_dir(D, e[FD], lam, mu, l2m, slw, r);
    h[VX] = slw * s[0] + r[VX]; h[VY] = slw * s[1] + r[VY]; h[VZ] = slw * s[2] + r[VZ];
    h[TXX] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]) + r[TXX];
    h[TYY] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]) + r[TYY];
    h[TZZ] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]) + r[TZZ];
    h[TXY] = mu * (G[0][1] + G[1][0]) + r[TXY];
    h[TXZ] = mu * (G[0][2] + G[2][0]) + r[TXZ];
    h[TYZ] = mu * (G[1][2] + G[2][1]) + r[TYZ];
#pragma unroll
    for (int c = 0; c < 9; c++) corr[c] = 0.f;
    if (a.pml[2 * FD].on) pml_face<MODE>(a, a.pml[2 * FD], FD, I, J, K, r, D, e[2], lam, mu, l2m, false, 0, corr);
    if (a.pml[2 * FD + 1].on) pml_face<MODE>(a, a.pml[2 * FD + 1], FD, I, J, K, r, D, e[2], lam, mu, l2m, false, 0, corr);
#pragma unroll
    for (int c = 0; c < 9; c++) h[c] += corr[c];
    rk_update<MODE>(a, p, v0, h);
    return;
  }

  // ---- shell and edges: PML edges and corners, rows under the free surface
  const int nk2 = g.nk + NG - 1;
  const bool top = (KIND == SHELL || KIND == TOP) && a.isfree && K >= nk2 - 3;
  const bool surfrow = (KIND == SHELL || KIND == TOP) && a.isfree && K == nk2;
  constexpr bool pml = KIND != TOP;
  const long fidx = ((long)J * g.nx + I) * 9;
  real corr[9], r[9], D[9], dvx[3], dvy[3];
#pragma unroll
  for (int c = 0; c < 9; c++) corr[c] = 0.f;
  // x
  derivs<ID>(w, v0, ox, D);
  dvx[0] = D[VX]; dvx[1] = D[VY]; dvx[2] = D[VZ];
  rhs_dir(D, e[0], lam, mu, l2m, slw, r);
#pragma unroll
  for (int c = 0; c < 9; c++) h[c] = r[c];
  if (pml && a.pml[0].on) pml_face<MODE>(a, a.pml[0], 0, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
  if (pml && a.pml[1].on) pml_face<MODE>(a, a.pml[1], 0, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
  // y
  derivs<JD>(w, v0, oy, D);
  dvy[0] = D[VX]; dvy[1] = D[VY]; dvy[2] = D[VZ];
  rhs_dir(D, e[1], lam, mu, l2m, slw, r);
#pragma unroll
  for (int c = 0; c < 9; c++) h[c] += r[c];
  if (pml && a.pml[2].on) pml_face<MODE>(a, a.pml[2], 1, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
  if (pml && a.pml[3].on) pml_face<MODE>(a, a.pml[3], 1, I, J, K, r, D, e[2], lam, mu, l2m, surfrow, fidx, corr);
  // z
  derivs<KD>(w, v0, oz, D);
  rhs_dir(D, e[2], lam, mu, l2m, slw, r);
  if (pml && a.pml[4].on) pml_face<MODE>(a, a.pml[4], 2, I, J, K, r, D, e[2], lam, mu, l2m, false, fidx, corr);
  if (pml && a.pml[5].on) pml_face<MODE>(a, a.pml[5], 2, I, J, K, r, D, e[2], lam, mu, l2m, false, fidx, corr);
  if (top && K >= nk2 - 2) {
    // velocity below the surface: the z part of the velocity gradient comes
    // from the conversion matrices (surface) or from 2nd / 4th order
    // one-sided differences (one / two rows below)
    const long sz = g.sz;
    real dz[3];
    if (K == nk2) {
      const real *X = a.free_mat + fidx;
      const real *Y = X + (long)g.ny * g.nx * 9;
      real o1[3], o2[3];
      mv3(X, dvx, o1); mv3(Y, dvy, o2);
      dz[0] = o1[0] + o2[0]; dz[1] = o1[1] + o2[1]; dz[2] = o1[2] + o2[2];
    } else if (K == nk2 - 1) {
      // velocities are components 0-2 of the first group: stride 4 floats
      const real *v = a.cur + 4 * p;
      dz[0] = mac22(v + VX, 4 * sz, KD); dz[1] = mac22(v + VY, 4 * sz, KD); dz[2] = mac22(v + VZ, 4 * sz, KD);
    } else {
      const real *v = a.cur + 4 * p;
      dz[0] = mac24(v + VX, 4 * sz, KD); dz[1] = mac24(v + VY, 4 * sz, KD); dz[2] = mac24(v + VZ, 4 * sz, KD);
    }
    real Dz[9], rz[9];
#pragma unroll
    for (int c = 0; c < 9; c++) Dz[c] = 0.f;
    Dz[VX] = dz[0]; Dz[VY] = dz[1]; Dz[VZ] = dz[2];
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
    const real *cur = a.cur;
    const long sy = g.sy;
    const real sj = slw / coef_jac(a.coef, p);
    // per tap the three traction rows at once; each row's sum over the
    // taps keeps the order of the coefficient table
    real dx[3] = { 0.f, 0.f, 0.f }, dy[3] = { 0.f, 0.f, 0.f }, dzz[3] = { 0.f, 0.f, 0.f };
    real t[3];
#pragma unroll
    for (int n = 0; n < 5; n++) {
      ctrac3(g, cur, a.coef, p + (ID ? n - 1 : n - 3), 0, t);
#pragma unroll
      for (int rr = 0; rr < 3; rr++) dx[rr] += wdrp<ID>(n) * t[rr];
    }
#pragma unroll
    for (int n = 0; n < 5; n++) {
      ctrac3(g, cur, a.coef, p + (JD ? n - 1 : n - 3) * sy, 1, t);
#pragma unroll
      for (int rr = 0; rr < 3; rr++) dy[rr] += wdrp<JD>(n) * t[rr];
    }
#pragma unroll
    for (int n = 0; n < 5; n++) {
      const int kk = K + (KD ? n - 1 : n - 3);
      if (kk == nk2) {
        t[0] = t[1] = t[2] = 0.f;
      } else {
        ctrac3(g, cur, a.coef, g.at(I, J, kk < nk2 ? kk : 2 * nk2 - kk), 2, t);
        if (kk > nk2) { t[0] = -t[0]; t[1] = -t[1]; t[2] = -t[2]; }
      }
#pragma unroll
      for (int rr = 0; rr < 3; rr++) dzz[rr] += wdrp<KD>(n) * t[rr];
    }
#pragma unroll
    for (int rr = 0; rr < 3; rr++) h[VX + rr] = (dx[rr] + dy[rr] + dzz[rr]) * sj;
  }
#pragma unroll
  for (int c = 0; c < 9; c++) h[c] += corr[c];
  rk_update<MODE>(a, p, v0, h);
}

template <int ID, int JD, int KD, int KIND>
void launch4(const VolArgs &a, int mode, cudaStream_t st) {
  if (a.nbox == 0) return;
  const dim3 blk(BX, BY, 1);
  dim3 grd(a.nblocks);
  if (KIND == INTERIOR) {
    const VolBox &B = a.box[0];
    const int nchunks = (B.nby + a.ychunk - 1) / a.ychunk;
    grd = dim3(B.nbx, a.ychunk, (B.k1 - B.k0 + 1) * nchunks);
  }
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

// This file is compiled once per kernel kind (CGFD_VOLUME_KIND = 0..7, set
// by the build) so that the 24 instantiations of each kind build in
// parallel; unit 0 also holds the host helpers.
#ifndef CGFD_VOLUME_KIND
#define CGFD_VOLUME_KIND 0
#endif

#if CGFD_VOLUME_KIND == 0
// boxes (interior indices, inclusive) -> block layout of one launch; with
// pack, boxes at most 24 points wide in x are packed (nbx = 0); the
// interior kernel's 3-D grid needs the tiled layout (pack = false)
void volume_boxes(VolArgs &a, const int (*boxes)[6], int n, bool pack) {
  a.nbox = 0;
  int first = 0;
  for (int q = 0; q < n; q++) {
    const int *b = boxes[q];
    if (b[1] < b[0] || b[3] < b[2] || b[5] < b[4]) continue;
    VolBox &B = a.box[a.nbox++];
    B.i0 = b[0]; B.i1 = b[1]; B.j0 = b[2]; B.j1 = b[3]; B.k0 = b[4]; B.k1 = b[5];
    const int ni = b[1] - b[0] + 1, nj = b[3] - b[2] + 1, nk = b[5] - b[4] + 1;
    if (pack && ni <= 24) {
      B.nbx = 0;
      B.nby = (ni * nj + BX * BY - 1) / (BX * BY);
      B.first = first;
      first += B.nby * nk;
    } else {
      B.nbx = (ni + BX - 1) / BX;
      B.nby = (nj + BY - 1) / BY;
      B.first = first;
      first += B.nbx * B.nby * nk;
    }
  }
  a.nblocks = first;
}

void launch_volume_interior(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<INTERIOR>(a, idir, jdir, kdir, mode, st);
}
#elif CGFD_VOLUME_KIND == 1
void launch_volume_shell(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<SHELL>(a, idir, jdir, kdir, mode, st);
}
#elif CGFD_VOLUME_KIND == 2
void launch_volume_face_x(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<FACE_X>(a, idir, jdir, kdir, mode, st);
}
#elif CGFD_VOLUME_KIND == 3
void launch_volume_face_y(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<FACE_Y>(a, idir, jdir, kdir, mode, st);
}
#elif CGFD_VOLUME_KIND == 4
void launch_volume_face_z(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<FACE_Z>(a, idir, jdir, kdir, mode, st);
}
#elif CGFD_VOLUME_KIND == 5
void launch_volume_edge(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<EDGE>(a, idir, jdir, kdir, mode, st);
}
#elif CGFD_VOLUME_KIND == 6
void launch_volume_plane(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<PLANE>(a, idir, jdir, kdir, mode, st);
}
#else
void launch_volume_top(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st) {
  launch_kind<TOP>(a, idir, jdir, kdir, mode, st);
}
#endif

}  // namespace cgfd
