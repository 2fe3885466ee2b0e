// fault.cu -- split-node fault kernels.
//
// Per RK stage the reference launches, per fault, wave2fault, the trial
// traction + slip-weakening friction kernel, fault2wave, the fault velocity
// RHS, the fault stress RHS (forward or backward variant), two fault RK
// updates, fault2wave again and the stage traction update, each as its own
// kernel (src/forward/drv_rk_curv_col.cu:277-588).  Here that becomes four
// kernels over the fault plane:
//
//   k_fault_weld    welded nodes: fault wavefield from the volume at i0
//                   (wave2fault_gpu, src/forward/transform.cu:101-212)
//   k_fault_trac    tractions J e . sigma of the stage input at the volume
//                   points i0-6..i0+6 around the split box, once each, into a
//                   per-fault scratch array read by the next two kernels
//   k_fault_split   split nodes, one thread each, in one pass:
//                   T1 traction image, trial traction and linear
//                   slip-weakening friction (trial_slipweakening_gpu,
//                   src/forward/trial_slipweakening.cu:92-388), stage
//                   traction output (fault_var_stage_update_gpu,
//                   fault_wav_t.cu:291-316), split-node velocity RHS
//                   (sv_curv_col_el_iso_fault_gpu.cu:323-429) and its RK
//                   update; then the velocity gradients of both sides and the
//                   fault traction rates with their RK update (..._stress_F_gpu
//                   :432-1159 / _B_gpu :1162-1879, split nodes), the
//                   split-node volume point of the output level from the
//                   fault fields (fault2wave_gpu, transform.cu:293-376) and,
//                   after the last stage, slip / slip rate / rupture time
//                   (fault_var_update_gpu, fault_wav_t.cu:198-264)
//   k_fault_slab    the volume points i0-3..i0+3 (not i0), one thread each:
//                   velocity RHS with the traction image through the fault
//                   (sv_curv_col_el_iso_rhs_fault_velo_gpu,
//                   src/forward/sv_curv_col_el_iso_fault_gpu.cu:192-322),
//                   stress RHS with the fault's one-sided operators
//                   (..._stress_F_gpu / _B_gpu, volume points) and the RK
//                   update of all nine components in whole 16-byte groups
//
// The volume stage kernel skips i0-3..i0+3 of split nodes, so these kernels
// own those points' RK update.  The slab and traction kernels give each
// (node, x offset) its own thread with the x offset fastest: the fault plane
// is a constant-x plane, so a warp over nodes alone would touch one cache
// line per thread on every volume access.
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

__device__ __forceinline__ long fidx(int c, int m, long ns, long nd) { return ((long)c * 2 + m) * ns + nd; }

// J * (e_d . sigma) at point q, 3 components (d: 0 xi, 1 eta, 2 zeta)
__device__ __forceinline__ void trac3(const Grid &g, const real *__restrict__ w, const real *__restrict__ cf,
                                      long q, int d, real t[3]) {
  const long sc = g.scmp;
  const real J = coef_jac(cf, q);
  const real4 e = coef_row(cf, sc, d, q);
  const real ex = e.x, ey = e.y, ez = e.z;
  // Txx ends the first 16-byte group, Tyy Tzz Tyz Txz are the second
  const real sxx = __ldg(w + g.w(TXX, q));
  const real4 s4 = __ldg(reinterpret_cast<const real4 *>(w + 4 * sc) + q);
  const real syy = s4.x, szz = s4.y, syz = s4.z, sxz = s4.w, sxy = __ldg(w + g.w(TXY, q));
  t[0] = J * (ex * sxx + ey * sxy + ez * sxz);
  t[1] = J * (ex * sxy + ey * syy + ez * syz);
  t[2] = J * (ex * sxz + ey * syz + ez * szz);
}

// odd extension of a 7-point line about its entry nf (3..6, the free
// surface): v[nf] = 0 and v[nf + l] = -v[nf - l] beyond it.  Fixed indices
// in every case keep the line in registers.
__device__ __forceinline__ void odd_image(real v[7], int nf) {
  switch (nf) {
    case 3: v[3] = 0.f; v[4] = -v[2]; v[5] = -v[1]; v[6] = -v[0]; break;
    case 4: v[4] = 0.f; v[5] = -v[3]; v[6] = -v[2]; break;
    case 5: v[5] = 0.f; v[6] = -v[4]; break;
    default: v[6] = 0.f; break;
  }
}

// stage update of N values; every level read is issued before the first
// store (the compiler cannot prove that the levels do not alias, and
// interleaved load / store pairs cost one memory round trip each)
template <int N>
__device__ __forceinline__ void rk_put_n(int mode, real ca, real cb, const real *cur, const real *pre,
                                         real *out, real *end, const long o[N], const real h[N]) {
  real u[N], e[N];
  if (mode == RK_FIRST) {
#pragma unroll
    for (int n = 0; n < N; n++) u[n] = cur[o[n]];
#pragma unroll
    for (int n = 0; n < N; n++) { out[o[n]] = u[n] + ca * h[n]; end[o[n]] = u[n] + cb * h[n]; }
  } else {
#pragma unroll
    for (int n = 0; n < N; n++) {
      if (mode == RK_MID) u[n] = pre[o[n]];
      e[n] = end[o[n]];
    }
#pragma unroll
    for (int n = 0; n < N; n++) {
      if (mode == RK_MID) out[o[n]] = u[n] + ca * h[n];
      end[o[n]] = e[n] + cb * h[n];
    }
  }
}

// slot of x offset d (-6..-1, 1..6) in the traction scratch
__device__ __forceinline__ int trac_slot(int d) { return d < 0 ? d + 6 : d + 5; }

// split-node volume point from the fault fields (fault2wave_gpu,
// transform.cu:293-376): velocity = mean of the two sides, stress from the
// traction vectors [T1 | mean T2 | mean T3] through the inverse metric.
__device__ void split_to_volume(const Grid &g, const real *__restrict__ cf, long sc, long ns, long nd,
                                int i0, int J, int K, const real *f, const real T1[3], real *wt) {
  const long p0 = g.at(i0, J, K);
  real mt[3][3];   // columns e_xi, e_eta, e_zeta
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const real4 e = coef_row(cf, sc, c, p0);
    mt[0][c] = e.x; mt[1][c] = e.y; mt[2][c] = e.z;
  }
  const real rj = 1.0f / coef_jac(cf, p0);
  real tr[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    tr[r][0] = T1[r];
    tr[r][1] = (f[fidx(FT2X + r, 0, ns, nd)] + f[fidx(FT2X + r, 1, ns, nd)]) * 0.5f;
    tr[r][2] = (f[fidx(FT3X + r, 0, ns, nd)] + f[fidx(FT3X + r, 1, ns, nd)]) * 0.5f;
  }
  const real c00 = mt[1][1] * mt[2][2] - mt[2][1] * mt[1][2], c01 = mt[2][1] * mt[0][2] - mt[0][1] * mt[2][2];
  const real c02 = mt[0][1] * mt[1][2] - mt[0][2] * mt[1][1], c10 = mt[1][2] * mt[2][0] - mt[1][0] * mt[2][2];
  const real c11 = mt[0][0] * mt[2][2] - mt[2][0] * mt[0][2], c12 = mt[1][0] * mt[0][2] - mt[0][0] * mt[1][2];
  const real c20 = mt[1][0] * mt[2][1] - mt[1][1] * mt[2][0], c21 = mt[2][0] * mt[0][1] - mt[0][0] * mt[2][1];
  const real c22 = mt[0][0] * mt[1][1] - mt[0][1] * mt[1][0];
  const real id = 1.0f / (c00 * mt[0][0] + c01 * mt[1][0] + c02 * mt[2][0]);
  const real mi[3][3] = { { c00 * id, c01 * id, c02 * id }, { c10 * id, c11 * id, c12 * id }, { c20 * id, c21 * id, c22 * id } };
  real st[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) st[r][c] = (tr[r][0] * mi[0][c] + tr[r][1] * mi[1][c] + tr[r][2] * mi[2][c]) * rj;
  real u[3];
#pragma unroll
  for (int c = 0; c < 3; c++) u[c] = (f[fidx(FVX + c, 0, ns, nd)] + f[fidx(FVX + c, 1, ns, nd)]) * 0.5f;
  reinterpret_cast<real4 *>(wt)[p0] = make_real4(u[0], u[1], u[2], st[0][0]);
  // the reference's fault2wave_gpu receives Tyz and Txz in swapped
  // positions (transform.cu:281-289 vs :293-300); kept for parity
  reinterpret_cast<real4 *>(wt + 4 * sc)[p0] =
      make_real4(st[1][1], st[2][2], (st[0][2] + st[2][0]) * 0.5f, (st[1][2] + st[2][1]) * 0.5f);
  wt[g.w(TXY, p0)] = (st[0][1] + st[1][0]) * 0.5f;
}

}  // namespace

// ---------------------------------------------------------------------------
__global__ void k_fault_weld(const FaultArgs a) {
  const Grid &g = a.g;
  const int j = a.wj0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int k = a.wk0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= a.wj0 + a.wnj || k >= a.wk0 + a.wnk) return;
  const int J = j + NG, K = k + NG;
  const long ns = (long)g.ny * g.nz, nd = J + (long)K * g.ny;
  if (a.F.flag[nd] & FL_SPLIT) return;
  const long p = g.at(a.F.i0, J, K);
  const real *w = a.wcur;
  real t2[3], t3[3];
  trac3(g, w, a.coef, p, 1, t2);
  trac3(g, w, a.coef, p, 2, t3);
  real *f = const_cast<real *>(a.fc);
#pragma unroll
  for (int m = 0; m < 2; m++) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      f[fidx(FVX + c, m, ns, nd)] = w[g.w(VX + c, p)];
      f[fidx(FT2X + c, m, ns, nd)] = t2[c];
      f[fidx(FT3X + c, m, ns, nd)] = t3[c];
    }
  }
}

// ---------------------------------------------------------------------------
// tractions of the stage input around the split box, one thread per
// (node, x offset), x offset fastest so that a warp reads contiguous x runs:
// T1 = J e_xi . sigma at x = i0+-1..6, T2 = J e_eta . sigma and
// T3 = J e_zeta . sigma at x = i0+-1..3.  The trial, friction and slab
// velocity kernels read them from here instead of recomputing each one
// (10 loads) for every tap.  Layout [9][tnk][tnj][12], x offset fastest.
__global__ void __launch_bounds__(192) k_fault_trac(const FaultArgs a) {
  const Grid &g = a.g;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long node = t / 12;
  if (node >= (long)a.tnj * a.tnk) return;
  const int slot = (int)(t - node * 12);
  const int d = slot < 6 ? slot - 6 : slot - 5;
  const int kk = (int)(node / a.tnj), jj = (int)(node - (long)kk * a.tnj);
  const long pl = (long)a.tnj * a.tnk * 12;
  const long q = g.at(a.F.i0 + d, a.tj0 + jj, a.tk0 + kk);
  real *tp = a.trac + node * 12 + slot;
  real v[3];
  trac3(g, a.wcur, a.coef, q, 0, v);
  tp[0] = v[0]; tp[pl] = v[1]; tp[2 * pl] = v[2];
  if (d >= -3 && d <= 3) {
    trac3(g, a.wcur, a.coef, q, 1, v);
    tp[3 * pl] = v[0]; tp[4 * pl] = v[1]; tp[5 * pl] = v[2];
    trac3(g, a.wcur, a.coef, q, 2, v);
    tp[6 * pl] = v[0]; tp[7 * pl] = v[1]; tp[8 * pl] = v[2];
  }
}

// ---------------------------------------------------------------------------
// split nodes, one thread per node: trial traction and linear slip-weakening
// friction (trial_slipweakening_gpu), the stage traction output, the refresh
// of the stage input's split-node volume point, and the split-node velocity
// RHS with its RK update
__device__ __forceinline__ void split_trial(const FaultArgs &a, int j, int k, uint8_t fl) {
  const Grid &g = a.g;
  const int J = j + NG, K = k + NG;
  const long ns = (long)g.ny * g.nz, nd = J + (long)K * g.ny, sc = g.scmp;
  const FaultDev &F = a.F;
  const int i0 = F.i0;
  const real *cf = a.coef;
  const long ny = g.ny;
  const int km = g.nk - (k + 1);
  const bool surf = a.isfree && km <= 3;
  const int nf = km + 3;

  // T1 = J e_xi . sigma at i0-3..i0+3 (index 3 is the split node, filled
  // after the friction law)
  real X1[7][3];
  const long pl = (long)a.tnj * a.tnk * 12;
  const real *tr = a.trac + ((long)(K - a.tk0) * a.tnj + (J - a.tj0)) * 12;
#pragma unroll
  for (int l = -3; l <= 3; l++) {
    if (l == 0) continue;
#pragma unroll
    for (int c = 0; c < 3; c++) X1[l + 3][c] = tr[c * pl + trac_slot(l)];
  }

  // along-fault derivatives of the fault tractions, both sides
  real DyT2[2][3], DzT3[2][3], R[2][3];
#pragma unroll
  for (int m = 0; m < 2; m++) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const real *t2 = a.fc + fidx(FT2X + c, m, ns, nd);
      DyT2[m][c] = (fl & FL_RUPY) ? mac22(t2, 1, a.jdir) : drp_rt(t2, 1, a.jdir);
      const real *t3 = a.fc + fidx(FT3X + c, m, ns, nd);
      real dz;
      if (surf) {
        // traction image of T3 about the free surface
        real v[7];
#pragma unroll
        for (int l = 0; l < 7; l++) v[l] = __ldg(t3 + (long)(l - 3) * ny);
        odd_image(v, nf);
        dz = drp_v(v + 3, a.kdir);
      } else {
        dz = (fl & FL_RUPZ) ? mac22(t3, ny, a.kdir) : drp_rt(t3, ny, a.kdir);
      }
      DzT3[m][c] = dz;
      const int s = 2 * m - 1;
      const real img = kA1 * X1[3 + s][c] + kA2 * X1[3 + 2 * s][c] + kA3 * X1[3 + 3 * s][c];
      R[m][c] = 0.5f * ((real)s * img + (DyT2[m][c] + DzT3[m][c]));
    }
  }

  // trial traction from the velocity jump of time level n and friction
  const long p0 = g.at(i0, J, K);
  const real jac0 = coef_jac(cf, p0);
  const real rho0 = F.scal[FS_RHO0 * ns + nd], rho1 = F.scal[FS_RHO1 * ns + nd];
  const real M0 = 0.5f * jac0 * rho0, M1 = 0.5f * jac0 * rho1;
  real Tr[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const real dV = a.fp[fidx(FVX + c, 1, ns, nd)] - a.fp[fidx(FVX + c, 0, ns, nd)];
    Tr[c] = 2.0f * (M0 * M1 * dV / a.dt + M0 * R[1][c] - M1 * R[0][c]) / (kA0 * (M0 + M1));
  }
  const real4 exi = coef_row(cf, sc, 0, p0);
  real vn[3] = { exi.x, exi.y, exi.z };
  const real vn0 = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
  const real jacvec = jac0 * vn0;
  vn[0] /= vn0; vn[1] /= vn0; vn[2] /= vn0;
  const real T0[3] = { F.scal[FS_T0X * ns + nd], F.scal[FS_T0Y * ns + nd], F.scal[FS_T0Z * ns + nd] };
  real Tl[3];
#pragma unroll
  for (int c = 0; c < 3; c++) Tl[c] = Tr[c] / jacvec + T0[c];
  const real Tn0 = Tl[0] * vn[0] + Tl[1] * vn[1] + Tl[2] * vn[2];
  real Ts[3] = { Tl[0] - vn[0] * Tn0, Tl[1] - vn[1] * Tn0, Tl[2] - vn[2] * Tn0 };
  const real Ts0 = sqrt(Ts[0] * Ts[0] + Ts[1] * Ts[1] + Ts[2] * Ts[2]);
  bool change = false;
  real Tau_n = Tn0;
  if (Tn0 >= 0.f) { Tau_n = 0.f; change = true; }     // the fault cannot open
  const real slip = F.out[CGFD_FAULT_SLIP * ns + nd];
  const real mus = F.scal[FS_MUS * ns + nd], mud = F.scal[FS_MUD * ns + nd];
  const real Dc = F.scal[FS_DC * ns + nd], C0 = F.scal[FS_C0 * ns + nd];
  const real fr = slip <= Dc ? mus - (mus - mud) * slip / Dc : mud;
  const real Tau_c = -fr * Tau_n + C0;
  real Tau_s = Ts0;
  if (Ts0 >= Tau_c) { Tau_s = Tau_c; change = true; }
  real Tau[3], T1s[3];
  if (change) {
    const real q = fabs(Ts0) < RL(1e-1) ? 0.f : Tau_s / Ts0;
#pragma unroll
    for (int c = 0; c < 3; c++) { Tau[c] = Tau_n * vn[c] + q * Ts[c]; T1s[c] = (Tau[c] - T0[c]) * jacvec; }
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) { Tau[c] = Tl[c]; T1s[c] = Tr[c]; }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) { F.scal[(FS_T1X + c) * ns + nd] = T1s[c]; X1[3][c] = T1s[c]; }
  // the stage input level sees the new split-node traction before the volume
  // kernel reads it (drv_rk_curv_col.cu:285, fault2wave on w_cur); no fault
  // kernel reads the volume at i0
  split_to_volume(g, cf, sc, ns, nd, i0, J, K, a.fc, T1s, const_cast<real *>(a.wcur));
  {
    const real s1[3] = { F.scal[FS_S1X * ns + nd], F.scal[FS_S1Y * ns + nd], F.scal[FS_S1Z * ns + nd] };
    const real s2[3] = { F.scal[FS_S2X * ns + nd], F.scal[FS_S2Y * ns + nd], F.scal[FS_S2Z * ns + nd] };
    const real tTs1 = Tau[0] * s1[0] + Tau[1] * s1[1] + Tau[2] * s1[2];
    const real tTs2 = Tau[0] * s2[0] + Tau[1] * s2[1] + Tau[2] * s2[2];
    real *Tn = F.out + CGFD_FAULT_TN * ns + nd, *T1o = F.out + CGFD_FAULT_TS1 * ns + nd, *T2o = F.out + CGFD_FAULT_TS2 * ns + nd;
    if (a.mode == RK_FIRST) { *Tn = a.rkb * Tau_n; *T1o = a.rkb * tTs1; *T2o = a.rkb * tTs2; }
    else { *Tn += a.rkb * Tau_n; *T1o += a.rkb * tTs1; *T2o += a.rkb * tTs2; }
  }

  // split-node velocity RHS and RK update (the output levels only; the
  // stress kernel of this stage reads the fault velocity of the input level)
  long o[6];
  real hv[6];
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const real rr = 1.0f / ((m ? rho1 : rho0) * jac0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const real dx = m == 0 ? (kA0 * X1[3][c] - kA1 * X1[2][c] - kA2 * X1[1][c] - kA3 * X1[0][c])
                              : (-kA0 * X1[3][c] + kA1 * X1[4][c] + kA2 * X1[5][c] + kA3 * X1[6][c]);
      hv[3 * m + c] = (dx + DyT2[m][c] + DzT3[m][c]) * rr;
      o[3 * m + c] = fidx(FVX + c, m, ns, nd);
    }
  }
  rk_put_n<6>(a.mode, a.ca, a.cb, a.fc, a.fp, a.fo, a.fe, o, hv);
}

// x offset from the fault of slab slot y = 0..5: -3, -2, -1, 1, 2, 3
__device__ __forceinline__ int slab_offset(int y) { return y < 3 ? y - 3 : y - 2; }

// slab work item t over the split box, six per node with the x offset
// fastest (a warp reads runs of contiguous x): node (j, k), offset s
__device__ __forceinline__ bool slab_item(const FaultArgs &a, long t, int &j, int &k, int &s) {
  const long node = t / 6;
  if (node >= (long)a.nj * a.nk) return false;
  const int r = (int)(t - node * 6);
  k = a.k0 + (int)(node / a.nj);
  j = a.j0 + (int)(node - (long)(k - a.k0) * a.nj);
  s = slab_offset(r);
  return true;
}

// ---------------------------------------------------------------------------
// velocity RHS at the six volume points i0-3..i0+3 (not i0) of split nodes,
// one thread per point, one warp per (slab offset, row of 32 nodes)
// (sv_curv_col_el_iso_rhs_fault_velo_gpu, :192-322)
__device__ __forceinline__ void slab_velocity(const FaultArgs &a, int j, int k, int s, real hv3[3]) {
  const Grid &g = a.g;
  const int J = j + NG, K = k + NG;
  const long ns = (long)g.ny * g.nz, nd = J + (long)K * g.ny, sc = g.scmp;
  const FaultDev &F = a.F;
  const int i0 = F.i0;
  const int km = g.nk - (k + 1);
  const bool surf = a.isfree && km <= 3;
  const int nf = km + 3;
  const long q = g.at(i0 + s, J, K);
  const long pl = (long)a.tnj * a.tnk * 12, row = (long)a.tnj * 12;
  const real *tr = a.trac + ((long)(K - a.tk0) * a.tnj + (J - a.tj0)) * 12;

  // T1 along x through this point: this side's volume points, the split
  // node's T1 at the fault, and beyond it the odd extension through the
  // split node (traction image)
  real v1[7][3];
#pragma unroll
  for (int l = -3; l <= 3; l++) {
    const int x = s + l;
    if (x == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) v1[l + 3][c] = F.scal[(FS_T1X + c) * ns + nd];
    } else if ((x < 0) == (s < 0)) {
#pragma unroll
      for (int c = 0; c < 3; c++) v1[l + 3][c] = tr[c * pl + trac_slot(x)];
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) v1[l + 3][c] = 0.f;
    }
  }
  real hv[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    real v[7];
#pragma unroll
    for (int l = 0; l < 7; l++) v[l] = v1[l][c];
    if (s == -2) { v[6] = 2.f * v[5] - v[4]; }
    if (s == -1) { v[5] = 2.f * v[4] - v[3]; v[6] = 2.f * v[4] - v[2]; }
    if (s == 1) { v[0] = 2.f * v[2] - v[4]; v[1] = 2.f * v[2] - v[3]; }
    if (s == 2) { v[0] = 2.f * v[1] - v[2]; }
    hv[c] = drp_v(v + 3, a.idir);
  }

  // y and z lines of T2 = J e_eta . sigma and T3 = J e_zeta . sigma
  const real *t2 = tr + 3 * pl + trac_slot(s), *t3 = t2 + 3 * pl;
  const real rr = coef_row(a.coef, sc, 2, q).w / coef_jac(a.coef, q);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    real y[7], z[7];
#pragma unroll
    for (int l = 0; l < 7; l++) {
      y[l] = t2[c * pl + (l - 3) * 12];
      z[l] = t3[c * pl + (l - 3) * row];
    }
    if (surf) {
      odd_image(z, nf);
    }
    hv3[c] = (hv[c] + drp_v(y + 3, a.jdir) + drp_v(z + 3, a.kdir)) * rr;
  }
}

// component c (0 x, 1 y, 2 z) of a 16-byte group
__device__ __forceinline__ real cmp3(const real4 &v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// drp, mac24 and mac22 (same weights, same order of the sums) of the three
// velocity components along stride st (in groups) from whole 16-byte groups
// (Vx Vy Vz Txx) of one level, direction f
__device__ __forceinline__ void vel_drp(const real4 *__restrict__ p, long st, int f, real o[3]) {
  if (f) {
    const real4 a = __ldg(p - st), b = __ldg(p), c = __ldg(p + st), d = __ldg(p + 2 * st), e = __ldg(p + 3 * st);
#pragma unroll
    for (int n = 0; n < 3; n++)
      o[n] = kC1 * cmp3(a, n) + kC2 * cmp3(b, n) + kC3 * cmp3(c, n) + kC4 * cmp3(d, n) + kC5 * cmp3(e, n);
  } else {
    const real4 a = __ldg(p + st), b = __ldg(p), c = __ldg(p - st), d = __ldg(p - 2 * st), e = __ldg(p - 3 * st);
#pragma unroll
    for (int n = 0; n < 3; n++)
      o[n] = -(kC1 * cmp3(a, n) + kC2 * cmp3(b, n) + kC3 * cmp3(c, n) + kC4 * cmp3(d, n) + kC5 * cmp3(e, n));
  }
}
__device__ __forceinline__ void vel_mac24(const real4 *__restrict__ p, long st, int f, real o[3]) {
  const real4 b = __ldg(p), c = __ldg(f ? p + st : p - st), d = __ldg(f ? p + 2 * st : p - 2 * st);
#pragma unroll
  for (int n = 0; n < 3; n++) {
    const real t = kB1 * cmp3(b, n) + kB2 * cmp3(c, n) + kB3 * cmp3(d, n);
    o[n] = f ? t : -t;
  }
}
__device__ __forceinline__ void vel_mac22(const real4 *__restrict__ p, long st, int f, real o[3]) {
  const real4 b = __ldg(p), c = __ldg(f ? p + st : p - st);
#pragma unroll
  for (int n = 0; n < 3; n++) o[n] = f ? cmp3(c, n) - cmp3(b, n) : cmp3(b, n) - cmp3(c, n);
}

// ---------------------------------------------------------------------------
// stress RHS and RK update at the six volume points i0-3..i0+3 (not i0) of
// split nodes, one thread per point, x offset fastest
// (sv_curv_col_el_iso_rhs_fault_stress_F_gpu :432-1159 / _B_gpu :1162-1879,
// volume points)
__device__ __forceinline__ void slab_stress(const FaultArgs &a, int j, int k, int s, real h[6]) {
  const Grid &g = a.g;
  const int J = j + NG, K = k + NG;
  const long ns = (long)g.ny * g.nz, nd = J + (long)K * g.ny, sc = g.scmp;
  const int i0 = a.F.i0;
  const real *w = a.wcur;
  const int km = g.nk - (k + 1);
  const bool fwd = a.idir == 1;
  const bool top = a.isfree && km == 0;
  // fault velocity of this side, input level
  real fV[3];
  const int m = s < 0 ? 0 : 1;
#pragma unroll
  for (int c = 0; c < 3; c++) fV[c] = a.fc[fidx(FVX + c, m, ns, nd)];
  const long q = g.at(i0 + s, J, K);
  // the velocity taps as whole 16-byte groups (Vx Vy Vz Txx): one load per
  // tap for all three components
  const real4 *V = reinterpret_cast<const real4 *>(w) + q;
  const real4 v0 = __ldg(V);
  real dx[3], dy[3], dz[3];
  if (fwd) {
    // forward operators; points left of the fault see the minus side
    if (s == 3) vel_drp(V, 1, 1, dx);
    else if (s == 2) vel_mac24(V, 1, 1, dx);
    else if (s == 1) vel_mac22(V, 1, 1, dx);
    else if (s == -1) {
#pragma unroll
      for (int c = 0; c < 3; c++) dx[c] = fV[c] - cmp3(v0, c);
    } else if (s == -2) {
      const real4 v1 = __ldg(V + 1);
#pragma unroll
      for (int c = 0; c < 3; c++) dx[c] = kB1 * cmp3(v0, c) + kB2 * cmp3(v1, c) + kB3 * fV[c];
    } else {
      const real4 vm = __ldg(V - 1), v1 = __ldg(V + 1), v2 = __ldg(V + 2);
#pragma unroll
      for (int c = 0; c < 3; c++)
        dx[c] = kC1 * cmp3(vm, c) + kC2 * cmp3(v0, c) + kC3 * cmp3(v1, c) + kC4 * cmp3(v2, c) + kC5 * fV[c];
    }
  } else {
    if (s == -3) vel_drp(V, 1, 0, dx);
    else if (s == -2) vel_mac24(V, 1, 0, dx);
    else if (s == -1) vel_mac22(V, 1, 0, dx);
    else if (s == 1) {
#pragma unroll
      for (int c = 0; c < 3; c++) dx[c] = cmp3(v0, c) - fV[c];
    } else if (s == 2) {
      const real4 vm = __ldg(V - 1);
#pragma unroll
      for (int c = 0; c < 3; c++) dx[c] = -(kB3 * fV[c] + kB2 * cmp3(vm, c) + kB1 * cmp3(v0, c));
    } else {
      const real4 vm2 = __ldg(V - 2), vm = __ldg(V - 1), v1 = __ldg(V + 1);
#pragma unroll
      for (int c = 0; c < 3; c++)
        dx[c] = -(kC5 * fV[c] + kC4 * cmp3(vm2, c) + kC3 * cmp3(vm, c) + kC2 * cmp3(v0, c) + kC1 * cmp3(v1, c));
    }
  }
  vel_drp(V, g.sy, a.jdir, dy);
  if (a.isfree && km == 1) vel_mac22(V, g.sz, a.kdir, dz);
  else if (a.isfree && km == 2) vel_mac24(V, g.sz, a.kdir, dz);
  else vel_drp(V, g.sz, a.kdir, dz);
  if (top) {
    const real *X = a.free_mat + ((long)J * g.nx + (i0 + s)) * 9;
    const real *Y = X + (long)g.ny * g.nx * 9;
    real o1[3], o2[3];
    mv3(X, dx, o1); mv3(Y, dy, o2);
#pragma unroll
    for (int c = 0; c < 3; c++) dz[c] = o1[c] + o2[c];
  }
  const real4 r0 = coef_row(a.coef, sc, 0, q), r1 = coef_row(a.coef, sc, 1, q), r2 = coef_row(a.coef, sc, 2, q);
  const real e[3][3] = { { r0.x, r0.y, r0.z }, { r1.x, r1.y, r1.z }, { r2.x, r2.y, r2.z } };
  const real lam = r0.w, mu = r1.w;
  const real l2m = lam + 2.0f * mu;
  real G[3][3];
#pragma unroll
  for (int b = 0; b < 3; b++)
#pragma unroll
    for (int c = 0; c < 3; c++) G[c][b] = e[0][b] * dx[c] + e[1][b] * dy[c] + e[2][b] * dz[c];
  h[0] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]);
  h[1] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]);
  h[2] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]);
  h[3] = mu * (G[1][2] + G[2][1]);   // Tyz
  h[4] = mu * (G[0][2] + G[2][0]);   // Txz
  h[5] = mu * (G[0][1] + G[1][0]);   // Txy
}

// ---------------------------------------------------------------------------
// split nodes, one thread per node: velocity gradients of both sides
// (continuity matrices or traction rate, free-surface rows), fault traction
// rates and their RK update, the split-node volume point of the output
// level, and after the last stage slip / slip rate / rupture time
// (sv_curv_col_el_iso_rhs_fault_stress_F_gpu :432-1159 / _B_gpu :1162-1879,
// split nodes; fault2wave_gpu; fault_var_update_gpu)
__device__ __forceinline__ void split_node(const FaultArgs &a, int j, int k, uint8_t fl) {
  const Grid &g = a.g;
  const int J = j + NG, K = k + NG;
  const long ns = (long)g.ny * g.nz, nd = J + (long)K * g.ny, sc = g.scmp;
  const FaultDev &F = a.F;
  const int i0 = F.i0;
  const real *w = a.wcur;
  const long ny = g.ny;
  const int km = g.nk - (k + 1);
  const bool fwd = a.idir == 1;
  const bool top = a.isfree && km == 0;
  // fault velocity of each side, input level: fV[m][c]
  real fV[2][3];
#pragma unroll
  for (int c = 0; c < 3; c++) { fV[0][c] = a.fc[fidx(FVX + c, 0, ns, nd)]; fV[1][c] = a.fc[fidx(FVX + c, 1, ns, nd)]; }

  // along-fault velocity derivatives of each side
  real Sx[2][3], Sy[2][3], Sz[2][3];
#pragma unroll
  for (int m = 0; m < 2; m++) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const real *v = a.fc + fidx(FVX + c, m, ns, nd);
      Sy[m][c] = (fl & FL_RUPY) ? mac22(v, 1, a.jdir) : drp_rt(v, 1, a.jdir);
      if (a.isfree && km == 1) Sz[m][c] = mac22(v, ny, a.kdir);
      else if (a.isfree && km == 2) Sz[m][c] = mac24(v, ny, a.kdir);
      else Sz[m][c] = (fl & FL_RUPZ) ? mac22(v, ny, a.kdir) : drp_rt(v, ny, a.kdir);
    }
  }
  const real *mat = F.mat;
  auto M = [&](int id) { return mat + ((long)id * ns + nd) * 9; };
  if (!top) {
    if (a.imethod == 1) {
      // one side from its one-sided difference, the other from continuity
      // of traction rate across the fault
      real o1[3], o2[3], o3[3], o4[3], o5[3];
      if (fwd) {
        const long q = g.at(i0 + 1, J, K);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[1][c] = w[g.w(VX + c, q)] - fV[1][c];
        mv3(M(FM_P2M1), Sx[1], o1); mv3(M(FM_P2M2), Sy[1], o2); mv3(M(FM_P2M3), Sz[1], o3);
        mv3(M(FM_P2M4), Sy[0], o4); mv3(M(FM_P2M5), Sz[0], o5);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[0][c] = o1[c] + o2[c] + o3[c] - o4[c] - o5[c];
      } else {
        const long q = g.at(i0 - 1, J, K);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[0][c] = fV[0][c] - w[g.w(VX + c, q)];
        mv3(M(FM_M2P1), Sx[0], o1); mv3(M(FM_M2P2), Sy[0], o2); mv3(M(FM_M2P3), Sz[0], o3);
        mv3(M(FM_M2P4), Sy[1], o4); mv3(M(FM_M2P5), Sz[1], o5);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[1][c] = o1[c] + o2[c] + o3[c] - o4[c] - o5[c];
      }
    } else {
      // normal derivative of each side from the traction rate
      real dt1[3] = { 0.f, 0.f, 0.f };
      if (fl & FL_GRID) { dt1[0] = F.scal[FS_HT1X * ns + nd]; dt1[1] = F.scal[FS_HT1Y * ns + nd]; dt1[2] = F.scal[FS_HT1Z * ns + nd]; }
      real o1[3], o2[3], o3[3];
      mv3(M(FM_T1VXPLUS), dt1, o1); mv3(M(FM_VYVXPLUS), Sy[1], o2); mv3(M(FM_VZVXPLUS), Sz[1], o3);
#pragma unroll
      for (int c = 0; c < 3; c++) Sx[1][c] = o1[c] - o2[c] - o3[c];
      mv3(M(FM_T1VXMIN), dt1, o1); mv3(M(FM_VYVXMIN), Sy[0], o2); mv3(M(FM_VZVXMIN), Sz[0], o3);
#pragma unroll
      for (int c = 0; c < 3; c++) Sx[0][c] = o1[c] - o2[c] - o3[c];
    }
  } else {
    // split nodes on the free surface: traction-free top as well
    auto FM = [&](int id) { return F.fmat + ((long)id * ny + J) * 9; };
    real o1[3], o2[3], o3[3];
    if (a.imethod == 1) {
      if (fwd) {
        const long q = g.at(i0 + 1, J, K);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[1][c] = w[g.w(VX + c, q)] - fV[1][c];
        mv3(FM(FF_P2M1), Sx[1], o1); mv3(FM(FF_P2M2), Sy[1], o2); mv3(FM(FF_P2M3), Sy[0], o3);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[0][c] = o1[c] + o2[c] - o3[c];
      } else {
        const long q = g.at(i0 - 1, J, K);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[0][c] = fV[0][c] - w[g.w(VX + c, q)];
        mv3(FM(FF_M2P1), Sx[0], o1); mv3(FM(FF_M2P2), Sy[0], o2); mv3(FM(FF_M2P3), Sy[1], o3);
#pragma unroll
        for (int c = 0; c < 3; c++) Sx[1][c] = o1[c] + o2[c] - o3[c];
      }
    } else {
      real dt1[3] = { 0.f, 0.f, 0.f };
      if (fl & FL_GRID) { dt1[0] = F.scal[FS_HT1X * ns + nd]; dt1[1] = F.scal[FS_HT1Y * ns + nd]; dt1[2] = F.scal[FS_HT1Z * ns + nd]; }
      mv3(FM(FF_T1VXPLUS), dt1, o1); mv3(FM(FF_VYVXPLUS), Sy[1], o2);
#pragma unroll
      for (int c = 0; c < 3; c++) Sx[1][c] = o1[c] - o2[c];
      mv3(FM(FF_T1VXMIN), dt1, o1); mv3(FM(FF_VYVXMIN), Sy[0], o2);
#pragma unroll
      for (int c = 0; c < 3; c++) Sx[0][c] = o1[c] - o2[c];
    }
    mv3(FM(FF_VX2VZ2), Sx[1], o1); mv3(FM(FF_VY2VZ2), Sy[1], o2);
#pragma unroll
    for (int c = 0; c < 3; c++) Sz[1][c] = o1[c] + o2[c];
    mv3(FM(FF_VX2VZ1), Sx[0], o1); mv3(FM(FF_VY2VZ1), Sy[0], o2);
#pragma unroll
    for (int c = 0; c < 3; c++) Sz[0][c] = o1[c] + o2[c];
  }

  // fault traction rates and RK update of T2, T3 on both sides
  {
    long o[12];
    real h[12];
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const int b2 = m ? FM_D21_2 : FM_D21_1, b3 = m ? FM_D31_2 : FM_D31_1;
      real g1[3], g2[3], g3[3];
      mv3(M(b2), Sx[m], g1); mv3(M(b2 + 1), Sy[m], g2); mv3(M(b2 + 2), Sz[m], g3);
#pragma unroll
      for (int c = 0; c < 3; c++) { h[6 * m + c] = g1[c] + g2[c] + g3[c]; o[6 * m + c] = fidx(FT2X + c, m, ns, nd); }
      mv3(M(b3), Sx[m], g1); mv3(M(b3 + 1), Sy[m], g2); mv3(M(b3 + 2), Sz[m], g3);
#pragma unroll
      for (int c = 0; c < 3; c++) { h[6 * m + 3 + c] = g1[c] + g2[c] + g3[c]; o[6 * m + 3 + c] = fidx(FT3X + c, m, ns, nd); }
    }
    rk_put_n<12>(a.mode, a.ca, a.cb, a.fc, a.fp, a.fo, a.fe, o, h);
  }

  // the split-node volume point of the output level from the fault fields
  {
    const bool last = a.mode == RK_LAST;
    const real T1s[3] = { F.scal[FS_T1X * ns + nd], F.scal[FS_T1Y * ns + nd], F.scal[FS_T1Z * ns + nd] };
    split_to_volume(g, a.coef, sc, ns, nd, i0, J, K, last ? a.fe : a.fo, T1s, last ? a.wend : a.wout);
  }

  // end of step: slip rate, slip, traction rate, peak slip rate, rupture time
  if (a.mode == RK_LAST) {
    const real *f = a.fe;
    const real s1[3] = { F.scal[FS_S1X * ns + nd], F.scal[FS_S1Y * ns + nd], F.scal[FS_S1Z * ns + nd] };
    const real s2[3] = { F.scal[FS_S2X * ns + nd], F.scal[FS_S2Y * ns + nd], F.scal[FS_S2Z * ns + nd] };
    real dV[3];
#pragma unroll
    for (int c = 0; c < 3; c++) dV[c] = f[fidx(FVX + c, 1, ns, nd)] - f[fidx(FVX + c, 0, ns, nd)];
    const real Vs1 = dV[0] * s1[0] + dV[1] * s1[1] + dV[2] * s1[2];
    const real Vs2 = dV[0] * s2[0] + dV[1] * s2[1] + dV[2] * s2[2];
    const real Vs = sqrt(Vs2 * Vs2 + Vs1 * Vs1);
    real *o = F.out;
    o[CGFD_FAULT_VS * ns + nd] = Vs;
    o[CGFD_FAULT_VS1 * ns + nd] = Vs1;
    o[CGFD_FAULT_VS2 * ns + nd] = Vs2;
    o[CGFD_FAULT_SLIP * ns + nd] += Vs * a.dt;
    o[CGFD_FAULT_SLIP1 * ns + nd] += Vs1 * a.dt;
    o[CGFD_FAULT_SLIP2 * ns + nd] += Vs2 * a.dt;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const real t1 = F.scal[(FS_T1X + c) * ns + nd];
      F.scal[(FS_HT1X + c) * ns + nd] = (t1 - F.scal[(FS_MT1X + c) * ns + nd]) / a.dt;
      F.scal[(FS_MT1X + c) * ns + nd] = t1;
    }
    if (Vs > o[CGFD_FAULT_PEAK_VS * ns + nd]) o[CGFD_FAULT_PEAK_VS * ns + nd] = Vs;
    uint8_t fl2 = F.flag[nd];
    if (!(fl2 & FL_T0SET) && Vs > RL(1e-3)) {
      o[CGFD_FAULT_INIT_T0 * ns + nd] = (a.ctl->it + 1) * a.dt;
      F.flag[nd] = fl2 | FL_T0SET;
    }
    if (!isfinite(Vs)) atomicOr(&a.ctl->err, 1);
  }
}

// ---------------------------------------------------------------------------
// split nodes, one thread per node: the trial traction and friction, then
// the traction rates, the split-node volume point of the output level and
// (after the last stage) slip and slip rate, in one pass.  The second part
// reads the traction this thread's first part wrote, the stage input at
// i0 +- 1 and the fault fields of the input level, none of which a split
// node's first part changes for another node, so one thread can do both.
__global__ void __launch_bounds__(128) k_fault_split(const FaultArgs a) {
  const int j = a.j0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int k = a.k0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= a.j0 + a.nj || k >= a.k0 + a.nk) return;
  const uint8_t fl = a.F.flag[(j + NG) + (long)(k + NG) * a.g.ny];
  if (!(fl & FL_SPLIT)) return;
  split_trial(a, j, k, fl);
  split_node(a, j, k, fl);
}

// the nine components of point p of a level (grouped layout)
__device__ __forceinline__ void lev9(const real *w, long sc, long p, real v[9]) {
  const real4 x = reinterpret_cast<const real4 *>(w)[p], y = reinterpret_cast<const real4 *>(w + 4 * sc)[p];
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
  v[8] = w[8 * sc + p];
}
// level value + c * h at point p, whole 16-byte groups
__device__ __forceinline__ void put9(real *w, long sc, long p, const real v[9], real c, const real h[9]) {
  reinterpret_cast<real4 *>(w)[p] = make_real4(v[0] + c * h[0], v[1] + c * h[1], v[2] + c * h[2], v[3] + c * h[3]);
  reinterpret_cast<real4 *>(w + 4 * sc)[p] =
      make_real4(v[4] + c * h[4], v[5] + c * h[5], v[6] + c * h[6], v[7] + c * h[7]);
  w[8 * sc + p] = v[8] + c * h[8];
}

// the six volume points i0-3..i0+3 (not i0) of split nodes, one thread per
// point with the x offset fastest: velocity RHS (traction image through the
// fault) and stress RHS (the fault's one-sided x operators), then the RK
// update of all nine components with whole-group stores
__global__ void __launch_bounds__(192) k_fault_slab(const FaultArgs a) {
  const Grid &g = a.g;
  int j, k, s;
  if (!slab_item(a, (long)blockIdx.x * blockDim.x + threadIdx.x, j, k, s)) return;
  if (!(a.F.flag[(j + NG) + (long)(k + NG) * g.ny] & FL_SPLIT)) return;
  real h[9];
  slab_velocity(a, j, k, s, h);
  slab_stress(a, j, k, s, h + 3);
  const long q = g.at(a.F.i0 + s, j + NG, k + NG), sc = g.scmp;
  real u[9], e[9];
  if (a.mode == RK_FIRST) {
    lev9(a.wcur, sc, q, u);
    put9(a.wout, sc, q, u, a.ca, h);
    put9(a.wend, sc, q, u, a.cb, h);
  } else {
    if (a.mode == RK_MID) lev9(a.wpre, sc, q, u);
    lev9(a.wend, sc, q, e);
    if (a.mode == RK_MID) put9(a.wout, sc, q, u, a.ca, h);
    put9(a.wend, sc, q, e, a.cb, h);
  }
}

// ---------------------------------------------------------------------------
// stations and fault stations of the current level (io_recv_keep,
// io_funcs.cu:428-469, including its use of corner 5 in place of corner 4;
// io_fault_recv_keep, io_funcs.cu:2313-2351)
__global__ void k_record(const StationArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int rec = a.ctl->nrec;
  const StationDev &S = a.st;
  if (rec >= S.max_rec) return;
  if (t < S.n * 9) {
    const int n = t / 9, c = t % 9;
    const long *ixp = S.idx + (long)n * 8;
    const real Lx2 = S.w[3 * n], Ly2 = S.w[3 * n + 1], Lz2 = S.w[3 * n + 2];
    const real Lx1 = 1.0f - Lx2, Ly1 = 1.0f - Ly2, Lz1 = 1.0f - Lz2;
    // component c of the level: points 4 floats apart in the grouped
    // arrays, 1 real apart for Txy
    const real *v = a.w + a.g.w(c, 0);
    const int u4 = wstep(c);
    const long ix[8] = { u4 * ixp[0], u4 * ixp[1], u4 * ixp[2], u4 * ixp[3],
                         u4 * ixp[4], u4 * ixp[5], u4 * ixp[6], u4 * ixp[7] };
    const real b0 = v[ix[0]], b1 = v[ix[1]], b2 = v[ix[2]], b3 = v[ix[3]];
    const real b5 = v[ix[5]], b6 = v[ix[6]], b7 = v[ix[7]];
    const real r = b0 * Lx1 * Ly1 * Lz1 + b1 * Lx2 * Ly1 * Lz1 + b2 * Lx1 * Ly2 * Lz1 + b3 * Lx2 * Ly2 * Lz1 +
                    b5 * Lx1 * Ly1 * Lz2 + b5 * Lx2 * Ly1 * Lz2 + b6 * Lx1 * Ly2 * Lz2 + b7 * Lx2 * Ly2 * Lz2;
    S.seis[(long)t * S.max_rec + rec] = r;
    if (!isfinite(r)) atomicOr(&a.ctl->err, 1);
  } else if (t < S.n * 9 + S.nf * 9) {
    const int u = t - S.n * 9, n = u / 9, c = u % 9;
    const real *o = a.fout[S.fid[n]] + (long)c * a.ns;
    const int *ix = S.fidx + 4 * n;
    const real Ly2 = S.fw[2 * n], Lz2 = S.fw[2 * n + 1], Ly1 = 1.0f - Ly2, Lz1 = 1.0f - Lz2;
    S.fseis[(long)u * S.max_rec + rec] = o[ix[0]] * Ly1 * Lz1 + o[ix[1]] * Ly2 * Lz1 + o[ix[2]] * Ly1 * Lz2 + o[ix[3]] * Ly2 * Lz2;
  }
}

__global__ void k_advance(Ctl *c, int max_rec) {
  c->it += 1;
  if (c->nrec < max_rec) c->nrec += 1;
}

// ---------------------------------------------------------------------------
// first part of a stage: welded nodes, tractions, trial traction and
// friction (which also refreshes the stage input at i0, read by the volume
// kernels); returns the number of launches
int launch_fault_pre(const FaultArgs &a, cudaStream_t st) {
  {
    dim3 blk(32, 4), grd((a.wnj + 31) / 32, (a.wnk + 3) / 4);
    k_fault_weld<<<grd, blk, 0, st>>>(a);
  }
  if (a.nj <= 0 || a.nk <= 0) return 1;
  {
    const long n = (long)a.tnj * a.tnk * 12;
    k_fault_trac<<<(unsigned)((n + 191) / 192), 192, 0, st>>>(a);
  }
  {
    dim3 blk(32, 4), grd((a.nj + 31) / 32, (a.nk + 3) / 4);
    k_fault_split<<<grd, blk, 0, st>>>(a);
  }
  return 3;
}

// second part: the slab points around the split nodes; independent of the
// volume kernels of the same stage (disjoint outputs, shared read-only input)
int launch_fault_post(const FaultArgs &a, cudaStream_t st) {
  if (a.nj <= 0 || a.nk <= 0) return 0;
  const long nslab = (long)a.nj * a.nk * 6;
  k_fault_slab<<<(unsigned)((nslab + 191) / 192), 192, 0, st>>>(a);
  return 1;
}

void launch_record(const StationArgs &a, cudaStream_t st) {
  const int n = (a.st.n + a.st.nf) * 9;
  if (n > 0 && a.st.max_rec > 0) k_record<<<(n + 127) / 128, 128, 0, st>>>(a);
}

void launch_advance(Ctl *c, int max_rec, cudaStream_t st) { k_advance<<<1, 1, 0, st>>>(c, max_rec); }

namespace {
// the interior nodes of the fault output fields [nf][ny*nz] into a
// contiguous [nf][nk][nj] array, so that one copy brings them to the host
__global__ void k_fault_gather(const real *__restrict__ out, real *__restrict__ dst, int nf, int nj, int nk,
                               int ny, long ns) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = (long)nj * nk;
  if (t >= n * nf) return;
  const int q = (int)(t / n);
  const long r = t - q * n;
  const int k = (int)(r / nj), j = (int)(r - (long)k * nj);
  dst[t] = __ldg(out + q * ns + (j + NG) + (long)(k + NG) * ny);
}
}  // namespace

void launch_fault_gather(const real *out, real *dst, int nf, const Grid &g, cudaStream_t st) {
  const long n = (long)nf * g.nj * g.nk;
  k_fault_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, dst, nf, g.nj, g.nk, g.ny, (long)g.ny * g.nz);
}

}  // namespace cgfd
