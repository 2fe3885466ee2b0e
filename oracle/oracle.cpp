/*
 * oracle.cpp -- CPU restatement of the reference's forward dynamic-rupture
 * path (hpc-lee/gpu-CGFD3D-dynamic).  TEST INFRASTRUCTURE: the checker for
 * the CUDA product, never part of it.
 *
 * Parity status: unpinned by reference outputs.  The reference has no tests,
 * no golden data and no CPU implementation; its code needs MPI, netCDF and a
 * GPU and is treated as unbuildable here.  Each routine below restates one
 * reference routine (file:line in its comment) loop by loop, keeping the
 * reference's evaluation order and its mixed float/double literal
 * arithmetic, and is checked by the known-answer tests in tests/.
 *
 * Layout follows the reference: 3 ghost points per side, x fastest,
 * iptr = i + j*nx + k*nx*ny; wavefield components Vx,Vy,Vz,Txx,Tyy,Tzz,Tyz,
 * Txz,Txy; four RK levels pre/tmp/rhs/end; fault wavefield
 * [side][Vx,Vy,Vz,T2x,T2y,T2z,T3x,T3y,T3z][nz][ny].
 *
 * Reference quirks kept on purpose (each is reproduced, not fixed):
 *  - fault2wave_gpu's parameter list names Txz/Tyz in the opposite order
 *    of its call (transform.cu:293 vs :281-289), so at split nodes the
 *    volume Tyz receives the xz stress and Txz the yz stress;
 *  - station trilinear weights use corner 5 twice, never corner 4
 *    (io_funcs.cu:452-461);
 *  - fault coefficients are built from rho before it becomes 1/rho
 *    (main_curv_col_el_3d.cu:544 vs :705);
 *  - wavefield ghosts stay zero (never written).
 */
#include "oracle.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_DOUBLE
typedef double real;
#else
typedef float real;
#endif

namespace {

thread_local std::string g_err;
int set_err(int code, const std::string &m) { g_err = m; return code; }

/* ---------------- operator tables (fd_t.cu:21-239, fd_t.h:9-140) ------- */

// DRP one-sided 5-point operator, stored exactly as mac_all_coef[3] (float)
const int  OP_IDX[2][5]  = { {-3, -2, -1, 0, 1}, {-1, 0, 1, 2, 3} };
const real OP_COEF[2][5] = {
  { (real)-0.041686285, (real)0.333411808, (real)-1.250117713, (real)0.666745142, (real)0.291647047 },
  { (real)-0.291647047, (real)-0.666745142, (real)1.250117713, (real)-0.333411808, (real)0.041686285 } };
// FD_Flags[8][3], 0 = backward, 1 = forward (fd_t.cu:146-159)
const int FD_FLAGS[8][3] = { {0,0,0},{1,1,0},{1,1,1},{0,0,1},{0,1,0},{1,0,0},{1,0,1},{0,1,1} };
const real RK_A[3] = { (real)0.5, (real)0.5, (real)1.0 };
const real RK_B[4] = { (real)(1.0/6.0), (real)(1.0/3.0), (real)(1.0/3.0), (real)(1.0/6.0) };

// macro constants, double literals as in fd_t.h
const double A0 = 1.2500392377, A1 = 1.5417647610, A2 = -0.3334118088, A3 = 0.0416862855;
const double B1 = -7.0/6.0, B2 = 8.0/6.0, B3 = -1.0/6.0;
const double C1 = -0.291647047, C2 = -0.666745142, C3 = 1.250117713, C4 = -0.333411808, C5 = 0.041686285;
const double D1 = -0.01666667, D2 = 0.15, D3 = -0.75, D5 = 0.75, D6 = -0.15, D7 = 0.01666667;

// M_FD_SHIFT_PTR_MAC22 / MAC24 / MACDRP on a pointer with stride
inline real mac22(const real *p, long s, int f) { return f ? (real)(p[s] - p[0]) : (real)(p[0] - p[-s]); }
inline real mac24(const real *p, long s, int f) {
  return f ? (real)((B1 * p[0]) + (B2 * p[s]) + (B3 * p[2*s]))
           : (real)(-(B1 * p[0]) - (B2 * p[-s]) - (B3 * p[-2*s]));
}
inline real macdrp(const real *p, long s, int f) {
  return f ? (real)((C1 * p[-s]) + (C2 * p[0]) + (C3 * p[s]) + (C4 * p[2*s]) + (C5 * p[3*s]))
           : (real)(-(C1 * p[s]) - (C2 * p[0]) - (C3 * p[-s]) - (C4 * p[-2*s]) - (C5 * p[-3*s]));
}
// M_FD_VEC (centre at v[0]) / M_FD_VEC_DRP (5 stored values) / VEC_24
inline real vec_c(const real *v, int f) {
  return f ? (real)((C1 * v[-1]) + (C2 * v[0]) + (C3 * v[1]) + (C4 * v[2]) + (C5 * v[3]))
           : (real)(-(C1 * v[1]) - (C2 * v[0]) - (C3 * v[-1]) - (C4 * v[-2]) - (C5 * v[-3]));
}
inline real vec_drp(const real *v, int f) {
  return f ? (real)((C1 * v[0]) + (C2 * v[1]) + (C3 * v[2]) + (C4 * v[3]) + (C5 * v[4]))
           : (real)(-(C5 * v[0]) - (C4 * v[1]) - (C3 * v[2]) - (C2 * v[3]) - (C1 * v[4]));
}
inline real vec24(const real *v, int f) {
  return f ? (real)((B1 * v[0]) + (B2 * v[1]) + (B3 * v[2]))
           : (real)(-(B3 * v[0]) - (B2 * v[1]) - (B1 * v[2]));
}
inline double center6(const real *p, long s) {
  return (D1 * p[-3*s]) + (D2 * p[-2*s]) + (D3 * p[-s]) + (D5 * p[s]) + (D6 * p[2*s]) + (D7 * p[3*s]);
}

/* ---------------- 3x3 helpers (src/lib/fdlib_math.cu:4-87) -------------- */
inline real norm3(const real *a) { real x2 = a[0]*a[0], y2 = a[1]*a[1], z2 = a[2]*a[2]; return std::sqrt(x2+y2+z2); }
inline void cross3(const real *a, const real *b, real *c) {
  c[0] = a[1]*b[2] - a[2]*b[1]; c[1] = a[2]*b[0] - a[0]*b[2]; c[2] = a[0]*b[1] - a[1]*b[0];
}
inline real dot3(const real *a, const real *b) { real r = 0; for (int i = 0; i < 3; i++) r += a[i]*b[i]; return r; }
void inv3(real m[3][3]) {
  double v[3][3];
  v[0][0] = m[1][1]*m[2][2] - m[2][1]*m[1][2];
  v[0][1] = m[2][1]*m[0][2] - m[0][1]*m[2][2];
  v[0][2] = m[0][1]*m[1][2] - m[0][2]*m[1][1];
  v[1][0] = m[1][2]*m[2][0] - m[1][0]*m[2][2];
  v[1][1] = m[0][0]*m[2][2] - m[2][0]*m[0][2];
  v[1][2] = m[1][0]*m[0][2] - m[0][0]*m[1][2];
  v[2][0] = m[1][0]*m[2][1] - m[1][1]*m[2][0];
  v[2][1] = m[2][0]*m[0][1] - m[0][0]*m[2][1];
  v[2][2] = m[0][0]*m[1][1] - m[0][1]*m[1][0];
  double det = v[0][0]*m[0][0] + v[0][1]*m[1][0] + v[0][2]*m[2][0];
  det = 1.0 / det;
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) m[i][j] = (real)(v[i][j] * det);
}
void mm3(const real a[3][3], const real b[3][3], real c[3][3]) {
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
    c[i][j] = 0; for (int k = 0; k < 3; k++) c[i][j] += a[i][k]*b[k][j];
  }
}
inline void mv3(const real a[3][3], const real *b, real *c) {
  c[0] = a[0][0]*b[0] + a[0][1]*b[1] + a[0][2]*b[2];
  c[1] = a[1][0]*b[0] + a[1][1]*b[1] + a[1][2]*b[2];
  c[2] = a[2][0]*b[0] + a[2][1]*b[1] + a[2][2]*b[2];
}
inline void load9(const real *src, real m[3][3]) { for (int q = 0; q < 9; q++) m[q/3][q%3] = src[q]; }
inline void store9(const real m[3][3], real *dst) { for (int q = 0; q < 9; q++) dst[q] = m[q/3][q%3]; }

// elastic traction-gradient block as written out in fault_coef_cal
// (fault_info.cu:180-300): D_ab = lam*ea(x)eb + mu*eb(x)ea + mu*(ea.eb) I
void dblock(const real *ea, const real *eb, real lam, real mu, real lam2mu, real d[3][3]) {
  d[0][0] = lam2mu*ea[0]*eb[0] + mu*(ea[1]*eb[1] + ea[2]*eb[2]);
  d[0][1] = lam*ea[0]*eb[1] + mu*ea[1]*eb[0];
  d[0][2] = lam*ea[0]*eb[2] + mu*ea[2]*eb[0];
  d[1][0] = mu*ea[0]*eb[1] + lam*ea[1]*eb[0];
  d[1][1] = lam2mu*ea[1]*eb[1] + mu*(ea[0]*eb[0] + ea[2]*eb[2]);
  d[1][2] = lam*ea[1]*eb[2] + mu*ea[2]*eb[1];
  d[2][0] = mu*ea[0]*eb[2] + lam*ea[2]*eb[0];
  d[2][1] = mu*ea[1]*eb[2] + lam*ea[2]*eb[1];
  d[2][2] = lam2mu*ea[2]*eb[2] + mu*(ea[0]*eb[0] + ea[1]*eb[1]);
}

enum { VX, VY, VZ, TXX, TYY, TZZ, TYZ, TXZ, TXY };
// fault wavefield component order (fault_wav_t.cu:96-150)
enum { FVX, FVY, FVZ, FT2X, FT2Y, FT2Z, FT3X, FT3Y, FT3Z };
enum { LPRE = 0, LTMP = 1, LRHS = 2, LEND = 3 };

struct PmlFace {
  int on = 0, L = 0;
  int i1, i2, j1, j2, k1, k2;      // region with ghosts (bdry_t.cu:118-151)
  int ni, nj, nk;
  size_t siz;                       // points of the face
  std::vector<real> A, B, D;        // per layer (L+1)
  std::vector<real> aux[4];         // 9*siz per level
  int lvl[4] = {0, 1, 2, 3};        // level indirection (pre/tmp/rhs/end)
  int cur = 0;                      // storage index of the stage's input level
  real *lev(int l) { return aux[lvl[l]].data(); }
};

struct Fault {
  int i0;                            // x index with ghosts
  int grid[4];                       // 0-based j1,j2,k1,k2
  // coefficients, [ny*nz*9] unless noted
  std::vector<real> D21_1, D22_1, D23_1, D31_1, D32_1, D33_1;
  std::vector<real> D21_2, D22_2, D23_2, D31_2, D32_2, D33_2;
  std::vector<real> M2P1, M2P2, M2P3, M2P4, M2P5, P2M1, P2M2, P2M3, P2M4, P2M5;
  std::vector<real> T1toVxMin, VytoVxMin, VztoVxMin, T1toVxPlus, VytoVxPlus, VztoVxPlus;
  std::vector<real> vec_n, vec_s1, vec_s2, x_et, y_et, z_et;   // [ny*nz*3] / [ny*nz]
  std::vector<real> rho_f;                                    // [2*ny*nz]
  // free-surface rows [ny*9]
  std::vector<real> Vx2Vz1, Vy2Vz1, Vx2Vz2, Vy2Vz2, P2M1f, P2M2f, P2M3f, M2P1f, M2P2f, M2P3f;
  std::vector<real> T1toVxfMin, VytoVxfMin, T1toVxfPlus, VytoVxfPlus;
  // inputs
  std::vector<real> T0x, T0y, T0z, mu_s, mu_d, Dc, C0;
  // outputs [11][ny*nz]
  std::vector<real> out;
  std::vector<real> tTn, tTs1, tTs2;
  std::vector<int> united, faultgrid, rup_y, rup_z, flag_rup, t0_flag;
  // wavefield: 4 levels x [2 sides][9][ny*nz]
  std::vector<real> fw[4];
  int lvl[4] = {0, 1, 2, 3};
  std::vector<real> T1x, T1y, T1z;      // [7][ny*nz]
  std::vector<real> hT1x, hT1y, hT1z, mT1x, mT1y, mT1z;
  real *lev(int l) { return fw[lvl[l]].data(); }
  real *o(int f) { return out.data() + (size_t)f * united.size(); }
};

struct Station { int i, j, k; real di, dj, dk; size_t idx[8]; };
struct FStation { int f; int j, k; real dj, dk; size_t idx[4]; };

} // namespace

struct oracle_solver {
  // grid
  int ni, nj, nk, nx, ny, nz;
  int ni1, ni2, nj1, nj2, nk1, nk2;
  size_t siz_iy, siz_iz, siz_icmp, siz_slice;
  real dt;
  int imethod, isfree;
  int it = 0;
  std::vector<real> x3d, y3d, z3d;
  std::vector<real> metric;   // 10 * siz_icmp: jac, xi_x, xi_y, xi_z, et_x.., zt_x..
  std::vector<real> lam, mu, rho;   // rho holds 1/rho after set-up
  std::vector<real> w[4];     // 4 levels of 9 * siz_icmp
  int wl[4] = {0, 1, 2, 3};
  PmlFace pml[3][2];
  int pml_on = 0;
  std::vector<real> matVx2Vz, matVy2Vz;   // [siz_iz*9]
  std::vector<Fault> faults;
  std::vector<Station> sta;
  std::vector<FStation> fsta;
  int max_rec = 0, nrec = 0;
  std::vector<real> seis, fseis;   // [n][9][max_rec]
  real dtmax = 0;
  // exponential sponge (bdryexp_t): masks along x, y, z and six blocks
  std::vector<real> abl_Ex, abl_Ey, abl_Ez;
  struct AblBlock { int enable, ni1, ni, nj1, nj, nk1, nk; } abl_blk[6];
  int abl_on = 0;
  // surface peaks [15][ny][nx] and displacement [3][ny][nx] (PG_d, Dis_accu_d)
  std::vector<real> pg, dis;

  size_t I(int i, int j, int k) const { return (size_t)i + (size_t)j*siz_iy + (size_t)k*siz_iz; }
  real *W(int l) { return w[wl[l]].data(); }
  real *M(int c) { return metric.data() + (size_t)c*siz_icmp; }
};

namespace {

/* -------- coordinates: gd_curv_gen_fault (gd_t.cu:402-545) ---------------- */
void geometric_symmetry(oracle_solver *S, real *v) {   // gd_t.cu:666-759
  const int nx = S->nx, ny = S->ny, nz = S->nz;
  const int ni1 = S->ni1, ni2 = S->ni2, nj1 = S->nj1, nj2 = S->nj2, nk1 = S->nk1, nk2 = S->nk2;
  for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) for (int i = 0; i < ni1; i++)
    v[S->I(i,j,k)] = 2*v[S->I(ni1,j,k)] - v[S->I(2*ni1-i,j,k)];
  for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) for (int i = ni2+1; i < nx; i++)
    v[S->I(i,j,k)] = 2*v[S->I(ni2,j,k)] - v[S->I(2*ni2-i,j,k)];
  for (int k = 0; k < nz; k++) for (int j = 0; j < nj1; j++) for (int i = 0; i < nx; i++)
    v[S->I(i,j,k)] = 2*v[S->I(i,nj1,k)] - v[S->I(i,2*nj1-j,k)];
  for (int k = 0; k < nz; k++) for (int j = nj2+1; j < ny; j++) for (int i = 0; i < nx; i++)
    v[S->I(i,j,k)] = 2*v[S->I(i,nj2,k)] - v[S->I(i,2*nj2-j,k)];
  for (int k = 0; k < nk1; k++) for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++)
    v[S->I(i,j,k)] = 2*v[S->I(i,j,nk1)] - v[S->I(i,j,2*nk1-k)];
  for (int k = nk2+1; k < nz; k++) for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++)
    v[S->I(i,j,k)] = 2*v[S->I(i,j,nk2)] - v[S->I(i,j,2*nk2-k)];
}

void gen_grid(oracle_solver *S, const cgfd_config *c) {
  S->x3d.assign(S->siz_icmp, 0); S->y3d.assign(S->siz_icmp, 0); S->z3d.assign(S->siz_icmp, 0);
  const int nj = S->nj, nk = S->nk;
  if (c->grid_mode == CGFD_GRID_IMPORT) {
    for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) for (int i = 0; i < S->ni; i++) {
      size_t src = (size_t)i + (size_t)S->ni*((size_t)j + (size_t)S->nj*k);
      size_t p = S->I(i+3, j+3, k+3);
      S->x3d[p] = c->x3d[src]; S->y3d[p] = c->y3d[src]; S->z3d[p] = c->z3d[src];
    }
  } else {
    const real dh = c->fault_interval;
    const size_t fsz = (size_t)nj*nk;
    auto FX = [&](int f, int j, int k) { return (real)c->fault_x[f*fsz + (size_t)(j-3) + (size_t)(k-3)*nj]; };
    auto FY = [&](int f, int j, int k) { return (real)c->fault_y[f*fsz + (size_t)(j-3) + (size_t)(k-3)*nj]; };
    auto FZ = [&](int f, int j, int k) { return (real)c->fault_z[f*fsz + (size_t)(j-3) + (size_t)(k-3)*nj]; };
    if (c->num_faults == 1) {
      int i0 = c->fault_x_index[0] - 1 + 3;
      for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++)
        for (int i = S->ni1; i <= S->ni2; i++) {
          size_t p = S->I(i,j,k);
          S->x3d[p] = FX(0,j,k) + (i-i0)*dh;
          S->y3d[p] = FY(0,j,k);
          S->z3d[p] = FZ(0,j,k);
        }
    } else {
      int i0 = c->fault_x_index[0] - 1 + 3;
      for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++) {
        real x = FX(0,j,k), y = FY(0,j,k), z = FZ(0,j,k);
        for (int i = S->ni1; i <= i0; i++) {
          size_t p = S->I(i,j,k); S->x3d[p] = x - (i0-i)*dh; S->y3d[p] = y; S->z3d[p] = z;
        }
      }
      for (int f = 1; f < c->num_faults; f++) {
        int ia = c->fault_x_index[f-1] - 1 + 3, ib = c->fault_x_index[f] - 1 + 3;
        for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++) {
          real x = FX(f,j,k), y = FY(f,j,k), z = FZ(f,j,k);
          size_t q = S->I(ia,j,k);
          real dhx = (x - S->x3d[q])/(ib-ia), dhy = (y - S->y3d[q])/(ib-ia), dhz = (z - S->z3d[q])/(ib-ia);
          for (int i = ia+1; i <= ib; i++) {
            size_t p = S->I(i,j,k);
            S->x3d[p] = x - (ib-i)*dhx; S->y3d[p] = y - (ib-i)*dhy; S->z3d[p] = z - (ib-i)*dhz;
          }
        }
      }
      int ib = c->fault_x_index[c->num_faults-1] - 1 + 3;
      for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++) {
        int f = c->num_faults-1;
        real x = FX(f,j,k), y = FY(f,j,k), z = FZ(f,j,k);
        for (int i = ib+1; i <= S->ni2; i++) {
          size_t p = S->I(i,j,k); S->x3d[p] = x + (i-ib)*dh; S->y3d[p] = y; S->z3d[p] = z;
        }
      }
    }
  }
  geometric_symmetry(S, S->x3d.data());
  geometric_symmetry(S, S->y3d.data());
  geometric_symmetry(S, S->z3d.data());
}

/* -------- metric: gd_curv_metric_cal (gd_t.cu:210-304) -------------------- */
void calc_metric(oracle_solver *S) {
  S->metric.assign(10*S->siz_icmp, 0);
  real *jac = S->M(0);
#pragma omp parallel for collapse(2)
  for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++)
    for (int i = S->ni1; i <= S->ni2; i++) {
      size_t p = S->I(i,j,k);
      const real *X = S->x3d.data() + p, *Y = S->y3d.data() + p, *Z = S->z3d.data() + p;
      long sy = (long)S->siz_iy, sz = (long)S->siz_iz;
      real v1[3] = { (real)center6(X,1), (real)center6(Y,1), (real)center6(Z,1) };
      real v2[3] = { (real)center6(X,sy), (real)center6(Y,sy), (real)center6(Z,sy) };
      real v3[3] = { (real)center6(X,sz), (real)center6(Y,sz), (real)center6(Z,sz) };
      real g[3];
      cross3(v1, v2, g);
      real J = dot3(g, v3);
      jac[p] = J;
      cross3(v2, v3, g); for (int q = 0; q < 3; q++) S->M(1+q)[p] = g[q] / J;
      cross3(v3, v1, g); for (int q = 0; q < 3; q++) S->M(4+q)[p] = g[q] / J;
      cross3(v1, v2, g); for (int q = 0; q < 3; q++) S->M(7+q)[p] = g[q] / J;
    }
  for (int c = 0; c < 10; c++) geometric_symmetry(S, S->M(c));
}

/* -------- time step limit: blk_dt_esti_curv (blk_t.cu:72-151) ------------ */
real dist_point2plane(const real *x0, const real *x1, const real *x2, const real *x3) {
  real x12[3] = { x2[0]-x1[0], x2[1]-x1[1], x2[2]-x1[2] };
  real x13[3] = { x3[0]-x1[0], x3[1]-x1[1], x3[2]-x1[2] };
  real p[3]; cross3(x12, x13, p);
  real d = dot3(p, x1);
  real L = (real)std::fabs(dot3(p, x0) - d);
  real P = norm3(p);
  return L / P;
}
void calc_dtmax(oracle_solver *S) {
  real best = (real)1.0e10;
#pragma omp parallel for collapse(2) reduction(min:best)
  for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++)
    for (int i = S->ni1; i <= S->ni2; i++) {
      size_t p = S->I(i,j,k);
      real Vp = std::sqrt((S->lam[p] + 2.0*S->mu[p]) / S->rho[p]);
      real dtLe = (real)1.0e20;
      real p0[3] = { S->x3d[p], S->y3d[p], S->z3d[p] };
      for (int kk = -1; kk <= 1; kk++) for (int jj = -1; jj <= 1; jj++) for (int ii = -1; ii <= 1; ii++) {
        if (ii != 0 && jj != 0 && kk != 0) {
          size_t a = p - ii, b = p - jj*S->siz_iy, c = p - kk*S->siz_iz;
          real p1[3] = { S->x3d[a], S->y3d[a], S->z3d[a] };
          real p2[3] = { S->x3d[b], S->y3d[b], S->z3d[b] };
          real p3[3] = { S->x3d[c], S->y3d[c], S->z3d[c] };
          real L = dist_point2plane(p0, p1, p2, p3);
          if (dtLe > L) dtLe = L;
        }
      }
      real dtp = (real)1.3 / Vp * dtLe;
      if (dtp < best) best = dtp;
    }
  S->dtmax = best;
}

/* -------- CFS-PML: bdry_pml_set (bdry_t.cu:80-251, 292-324, 327-440) ---- */
void pml_set(oracle_solver *S, const cgfd_config *c) {
  const float CONSPD = 2.0f, CONSPB = 2.0f, CONSPA = 1.0f;
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
    PmlFace &F = S->pml[d][s];
    F.on = c->pml_layers[d][s] > 0;
    F.L = F.on ? c->pml_layers[d][s] : 0;
    F.i1 = S->ni1; F.i2 = S->ni2; F.j1 = S->nj1; F.j2 = S->nj2; F.k1 = S->nk1; F.k2 = S->nk2;
    if (d == 0 && s == 0) F.i2 = S->ni1 + F.L;
    if (d == 0 && s == 1) F.i1 = S->ni2 - F.L;
    if (d == 1 && s == 0) F.j2 = S->nj1 + F.L;
    if (d == 1 && s == 1) F.j1 = S->nj2 - F.L;
    if (d == 2 && s == 0) F.k2 = S->nk1 + F.L;
    if (d == 2 && s == 1) F.k1 = S->nk2 - F.L;
    if (!F.on) continue;
    S->pml_on = 1;
    F.ni = F.i2 - F.i1 + 1; F.nj = F.j2 - F.j1 + 1; F.nk = F.k2 - F.k1 + 1;
    F.siz = (size_t)F.ni*F.nj*F.nk;
    // average spacing and length along the normal (bdry_cal_abl_len_dh)
    double Lsum = 0.0; int num = 0;
    auto seg = [&](size_t a, size_t b) {
      double x0 = S->x3d[a], y0 = S->y3d[a], z0 = S->z3d[a];
      double x1 = S->x3d[b], y1 = S->y3d[b], z1 = S->z3d[b];
      Lsum += std::sqrt((x1-x0)*(x1-x0) + (y1-y0)*(y1-y0) + (z1-z0)*(z1-z0)); num += 1;
    };
    float avg_dh, avg_L;
    if (d == 0) {
      for (int k = F.k1; k <= F.k2; k++) for (int j = F.j1; j <= F.j2; j++)
        for (int i = F.i1+1; i <= F.i2; i++) seg(S->I(i-1,j,k), S->I(i,j,k));
      avg_dh = (float)(Lsum/num); avg_L = avg_dh * (F.i2 - F.i1);
    } else if (d == 1) {
      for (int k = F.k1; k <= F.k2; k++) for (int i = F.i1; i <= F.i2; i++)
        for (int j = F.j1+1; j <= F.j2; j++) seg(S->I(i,j-1,k), S->I(i,j,k));
      avg_dh = (float)(Lsum/num); avg_L = avg_dh * (F.j2 - F.j1);
    } else {
      for (int j = F.j1; j <= F.j2; j++) for (int i = F.i1; i <= F.i2; i++)
        for (int k = F.k1+1; k <= F.k2; k++) seg(S->I(i,j,k-1), S->I(i,j,k));
      avg_dh = (float)(Lsum/num); avg_L = avg_dh * (F.k2 - F.k1);
    }
    int npoints = F.L + 1;
    float num_lay = (float)(npoints - 1);
    float Rpp = (float)(std::pow(10, -((std::log10((double)num_lay) - 1.0)/std::log10(2.0) + 4.0)));
    float Vp = c->pml_ref_vel[d][s];
    float dmax = (float)(-Vp / (2.0 * avg_L) * std::log(Rpp) * (CONSPD + 1.0));
    float amax = c->pml_alpha_max[d][s], bmax = c->pml_beta_max[d][s];
    F.A.assign(npoints, 0); F.B.assign(npoints, 0); F.D.assign(npoints, 0);
    for (int n = 0; n < npoints; n++) {
      float L = n * avg_dh;
      int i = (s == 0) ? npoints - 1 - n : n;
      float xl = L / avg_L;
      float Dv = (L < 0) ? 0.0f : (float)(dmax * std::pow(xl, CONSPD));
      float Av = (L < 0) ? 0.0f : (float)(amax * (1.0 - std::pow(xl, CONSPA)));
      float Bv = (L < 0) ? 1.0f : (float)(1.0 + (bmax - 1.0) * std::pow(xl, CONSPB));
      Dv /= Bv;
      Av += Dv;
      Bv = (float)(1.0 / Bv);
      F.D[i] = Dv; F.A[i] = Av; F.B[i] = Bv;
    }
    for (int l = 0; l < 4; l++) F.aux[l].assign(9*F.siz, 0);
  }
}

/* -------- free-surface conversion: sv_curv_col_el_iso_dvh2dvz_gpu
 *          (sv_curv_col_el_iso_gpu.cu:1297-1405) ------------------------- */
void free_set(oracle_solver *S) {
  S->matVx2Vz.assign(S->siz_iz*9, 0); S->matVy2Vz.assign(S->siz_iz*9, 0);
  int k = S->nk2;
  for (int j = S->nj1; j <= S->nj2; j++) for (int i = S->ni1; i <= S->ni2; i++) {
    size_t p = S->I(i,j,k);
    real e11 = S->M(1)[p], e12 = S->M(2)[p], e13 = S->M(3)[p];
    real e21 = S->M(4)[p], e22 = S->M(5)[p], e23 = S->M(6)[p];
    real e31 = S->M(7)[p], e32 = S->M(8)[p], e33 = S->M(9)[p];
    real la = S->lam[p], mu = S->mu[p];
    real l2m = la + 2.0f*mu;
    real A[3][3], B[3][3], C[3][3], AB[3][3], AC[3][3];
    A[0][0] = l2m*e31*e31 + mu*(e32*e32+e33*e33);
    A[0][1] = la*e31*e32 + mu*e32*e31;
    A[0][2] = la*e31*e33 + mu*e33*e31;
    A[1][0] = la*e32*e31 + mu*e31*e32;
    A[1][1] = l2m*e32*e32 + mu*(e31*e31+e33*e33);
    A[1][2] = la*e32*e33 + mu*e33*e32;
    A[2][0] = la*e33*e31 + mu*e31*e33;
    A[2][1] = la*e33*e32 + mu*e32*e33;
    A[2][2] = l2m*e33*e33 + mu*(e31*e31+e32*e32);
    inv3(A);
    B[0][0] = -l2m*e31*e11 - mu*(e32*e12+e33*e13);
    B[0][1] = -la*e31*e12 - mu*e32*e11;
    B[0][2] = -la*e31*e13 - mu*e33*e11;
    B[1][0] = -la*e32*e11 - mu*e31*e12;
    B[1][1] = -l2m*e32*e12 - mu*(e31*e11+e33*e13);
    B[1][2] = -la*e32*e13 - mu*e33*e12;
    B[2][0] = -la*e33*e11 - mu*e31*e13;
    B[2][1] = -la*e33*e12 - mu*e32*e13;
    B[2][2] = -l2m*e33*e13 - mu*(e31*e11+e32*e12);
    C[0][0] = -l2m*e31*e21 - mu*(e32*e22+e33*e23);
    C[0][1] = -la*e31*e22 - mu*e32*e21;
    C[0][2] = -la*e31*e23 - mu*e33*e21;
    C[1][0] = -la*e32*e21 - mu*e31*e22;
    C[1][1] = -l2m*e32*e22 - mu*(e31*e21+e33*e23);
    C[1][2] = -la*e32*e23 - mu*e33*e22;
    C[2][0] = -la*e33*e21 - mu*e31*e23;
    C[2][1] = -la*e33*e22 - mu*e32*e23;
    C[2][2] = -l2m*e33*e23 - mu*(e31*e21+e32*e22);
    mm3(A, B, AB); mm3(A, C, AC);
    size_t ij = ((size_t)j*S->siz_iy + i)*9;
    store9(AB, &S->matVx2Vz[ij]); store9(AC, &S->matVy2Vz[ij]);
  }
}

/* -------- fault coefficients: fault_coef_cal (fault_info.cu:98-850) ----- */
void fault_coef(oracle_solver *S, Fault &F) {
  const size_t ns = S->siz_slice;
  auto a9 = [&](std::vector<real> &v) { v.assign(ns*9, 0); };
  a9(F.D21_1); a9(F.D22_1); a9(F.D23_1); a9(F.D31_1); a9(F.D32_1); a9(F.D33_1);
  a9(F.D21_2); a9(F.D22_2); a9(F.D23_2); a9(F.D31_2); a9(F.D32_2); a9(F.D33_2);
  a9(F.M2P1); a9(F.M2P2); a9(F.M2P3); a9(F.M2P4); a9(F.M2P5);
  a9(F.P2M1); a9(F.P2M2); a9(F.P2M3); a9(F.P2M4); a9(F.P2M5);
  a9(F.T1toVxMin); a9(F.VytoVxMin); a9(F.VztoVxMin); a9(F.T1toVxPlus); a9(F.VytoVxPlus); a9(F.VztoVxPlus);
  F.vec_n.assign(ns*3, 0); F.vec_s1.assign(ns*3, 0); F.vec_s2.assign(ns*3, 0);
  F.x_et.assign(ns, 0); F.y_et.assign(ns, 0); F.z_et.assign(ns, 0);
  F.rho_f.assign(2*ns, 0);
  auto af = [&](std::vector<real> &v) { v.assign((size_t)S->ny*9, 0); };
  af(F.Vx2Vz1); af(F.Vy2Vz1); af(F.Vx2Vz2); af(F.Vy2Vz2); af(F.P2M1f); af(F.P2M2f); af(F.P2M3f);
  af(F.M2P1f); af(F.M2P2f); af(F.M2P3f); af(F.T1toVxfMin); af(F.VytoVxfMin); af(F.T1toVxfPlus); af(F.VytoVxfPlus);

  for (int k = 0; k < S->nz; k++) for (int j = 0; j < S->ny; j++) {
    size_t p = S->I(F.i0, j, k), pf = (size_t)j + (size_t)k*S->ny;
    real rho = S->rho[p], mu = S->mu[p], lam = S->lam[p];
    real l2m = lam + 2.0*mu;
    real jac = S->M(0)[p];
    real e1[3] = { S->M(1)[p], S->M(2)[p], S->M(3)[p] };
    real e2[3] = { S->M(4)[p], S->M(5)[p], S->M(6)[p] };
    real e3[3] = { S->M(7)[p], S->M(8)[p], S->M(9)[p] };
    F.rho_f[pf] = rho; F.rho_f[pf + ns] = rho;
    real D11_1[3][3], D12_1[3][3], D13_1[3][3], D11_2[3][3], D12_2[3][3], D13_2[3][3];
    real t[3][3];
    dblock(e1, e1, lam, mu, l2m, D11_1); dblock(e1, e2, lam, mu, l2m, D12_1); dblock(e1, e3, lam, mu, l2m, D13_1);
    dblock(e1, e1, lam, mu, l2m, D11_2); dblock(e1, e2, lam, mu, l2m, D12_2); dblock(e1, e3, lam, mu, l2m, D13_2);
    const real *ea[3] = { e1, e2, e3 };
    std::vector<real> *side1[2][3] = { { &F.D21_1, &F.D22_1, &F.D23_1 }, { &F.D31_1, &F.D32_1, &F.D33_1 } };
    std::vector<real> *side2[2][3] = { { &F.D21_2, &F.D22_2, &F.D23_2 }, { &F.D31_2, &F.D32_2, &F.D33_2 } };
    for (int a = 0; a < 2; a++) for (int b = 0; b < 3; b++) {
      dblock(ea[a+1], ea[b], lam, mu, l2m, t); store9(t, &(*side1[a][b])[pf*9]);
      dblock(ea[a+1], ea[b], lam, mu, l2m, t); store9(t, &(*side2[a][b])[pf*9]);
    }
    for (int q = 0; q < 9; q++) {
      int ii = q/3, jj = q%3;
      D11_1[ii][jj] *= jac; D12_1[ii][jj] *= jac; D13_1[ii][jj] *= jac;
      D11_2[ii][jj] *= jac; D12_2[ii][jj] *= jac; D13_2[ii][jj] *= jac;
      for (int a = 0; a < 2; a++) for (int b = 0; b < 3; b++) {
        (*side1[a][b])[pf*9+q] *= jac; (*side2[a][b])[pf*9+q] *= jac;
      }
    }
    real m1[3][3], m2[3][3];
    // method 1, minus -> plus
    std::memcpy(m1, D11_2, sizeof(m1)); inv3(m1);
    mm3(m1, D11_1, m2); store9(m2, &F.M2P1[pf*9]);
    mm3(m1, D12_1, m2); store9(m2, &F.M2P2[pf*9]);
    mm3(m1, D13_1, m2); store9(m2, &F.M2P3[pf*9]);
    mm3(m1, D12_2, m2); store9(m2, &F.M2P4[pf*9]);
    mm3(m1, D13_2, m2); store9(m2, &F.M2P5[pf*9]);
    // plus -> minus
    std::memcpy(m1, D11_1, sizeof(m1)); inv3(m1);
    mm3(m1, D11_2, m2); store9(m2, &F.P2M1[pf*9]);
    mm3(m1, D12_2, m2); store9(m2, &F.P2M2[pf*9]);
    mm3(m1, D13_2, m2); store9(m2, &F.P2M3[pf*9]);
    mm3(m1, D12_1, m2); store9(m2, &F.P2M4[pf*9]);
    mm3(m1, D13_1, m2); store9(m2, &F.P2M5[pf*9]);
    // method 2
    std::memcpy(m1, D11_1, sizeof(m1)); inv3(m1);
    store9(m1, &F.T1toVxMin[pf*9]);
    mm3(m1, D12_1, m2); store9(m2, &F.VytoVxMin[pf*9]);
    mm3(m1, D13_1, m2); store9(m2, &F.VztoVxMin[pf*9]);
    std::memcpy(m1, D11_2, sizeof(m1)); inv3(m1);
    store9(m1, &F.T1toVxPlus[pf*9]);
    mm3(m1, D12_2, m2); store9(m2, &F.VytoVxPlus[pf*9]);
    mm3(m1, D13_2, m2); store9(m2, &F.VztoVxPlus[pf*9]);
    // base vectors
    real m3[3][3] = { {e1[0], e1[1], e1[2]}, {e2[0], e2[1], e2[2]}, {e3[0], e3[1], e3[2]} };
    inv3(m3);
    F.x_et[pf] = m3[0][1]; F.y_et[pf] = m3[1][1]; F.z_et[pf] = m3[2][1];
    real s1[3] = { m3[0][1], m3[1][1], m3[2][1] };
    real nrm = norm3(s1); for (int q = 0; q < 3; q++) s1[q] /= nrm;
    real vn[3] = { e1[0], e1[1], e1[2] };
    nrm = norm3(vn); for (int q = 0; q < 3; q++) vn[q] /= nrm;
    real s2[3]; cross3(vn, s1, s2);
    for (int q = 0; q < 3; q++) { F.vec_n[pf*3+q] = vn[q]; F.vec_s1[pf*3+q] = s1[q]; F.vec_s2[pf*3+q] = s2[q]; }

    if (k == S->nk2) {   // (k-3+gnk1) == total_point_z-1 on one rank
      real A[3][3], B[3][3], C[3][3], Vx2Vz1[3][3], Vy2Vz1[3][3], Vx2Vz2[3][3], Vy2Vz2[3][3];
      for (int q = 0; q < 9; q++) {
        A[q/3][q%3] = F.D33_1[pf*9+q]; B[q/3][q%3] = -F.D31_1[pf*9+q]; C[q/3][q%3] = -F.D32_1[pf*9+q];
      }
      inv3(A); mm3(A, B, Vx2Vz1); mm3(A, C, Vy2Vz1);
      for (int q = 0; q < 9; q++) {
        A[q/3][q%3] = F.D33_2[pf*9+q]; B[q/3][q%3] = -F.D31_2[pf*9+q]; C[q/3][q%3] = -F.D32_2[pf*9+q];
      }
      inv3(A); mm3(A, B, Vx2Vz2); mm3(A, C, Vy2Vz2);
      real un[3] = { e1[0], e1[1], e1[2] };
      real us1[3] = { F.x_et[pf], F.y_et[pf], F.z_et[pf] };
      real us2[3]; cross3(un, us1, us2);
      nrm = norm3(us2); for (int q = 0; q < 3; q++) us2[q] /= nrm;
      real g1 = 0.0, g2 = 0.0, g3 = 0.0;
      real h1 = us2[0]*e1[0] + us2[1]*e1[1] + us2[2]*e1[2];
      real h2 = us2[0]*e2[0] + us2[1]*e2[1] + us2[2]*e2[2];
      real h3 = us2[0]*e3[0] + us2[1]*e3[1] + us2[2]*e3[2];
      nrm = norm3(un); h1 = h1/nrm; h2 = h2/nrm; h3 = h3/nrm;
      real D11_1f[3][3], D12_1f[3][3], D13_1f[3][3], D11_2f[3][3], D12_2f[3][3], D13_2f[3][3];
      for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) {
        real To1 = us1[ii]*un[jj], To2 = us2[ii]*un[jj];
        real a12 = mu*g1*To1, b12 = mu*g2*To1, c12 = mu*g3*To1;
        real a13 = mu*h1*To2, b13 = mu*h2*To2, c13 = mu*h3*To2;
        D11_1f[ii][jj] = D11_1[ii][jj] + a12 + a13;
        D12_1f[ii][jj] = D12_1[ii][jj] + b12 + b13;
        D13_1f[ii][jj] = D13_1[ii][jj] + c12 + c13;
        D11_2f[ii][jj] = D11_2[ii][jj] + a12 + a13;
        D12_2f[ii][jj] = D12_2[ii][jj] + b12 + b13;
        D13_2f[ii][jj] = D13_2[ii][jj] + c12 + c13;
      }
      real t1[3][3], t2[3][3], t3[3][3], t4[3][3];
      mm3(D13_1f, Vx2Vz1, t1); mm3(D13_1f, Vy2Vz1, t2); mm3(D13_2f, Vx2Vz2, t3); mm3(D13_2f, Vy2Vz2, t4);
      real Vx1f[3][3], Vy1f[3][3], Vx2f[3][3], Vy2f[3][3];
      for (int ii = 0; ii < 3; ii++) for (int jj = 0; jj < 3; jj++) {
        Vx1f[ii][jj] = D11_1f[ii][jj] + t1[ii][jj]; Vy1f[ii][jj] = D12_1f[ii][jj] + t2[ii][jj];
        Vx2f[ii][jj] = D11_2f[ii][jj] + t3[ii][jj]; Vy2f[ii][jj] = D12_2f[ii][jj] + t4[ii][jj];
      }
      real To[3][3], P1[3][3], P2[3][3], P3[3][3], Q1[3][3], Q2[3][3], Q3[3][3];
      std::memcpy(To, Vx1f, sizeof(To)); inv3(To);
      mm3(To, Vx2f, P1); mm3(To, Vy2f, P2); mm3(To, Vy1f, P3);
      store9(To, &F.T1toVxfMin[(size_t)j*9]); store9(P3, &F.VytoVxfMin[(size_t)j*9]);
      std::memcpy(To, Vx2f, sizeof(To)); inv3(To);
      mm3(To, Vx1f, Q1); mm3(To, Vy1f, Q2); mm3(To, Vy2f, Q3);
      store9(To, &F.T1toVxfPlus[(size_t)j*9]); store9(Q3, &F.VytoVxfPlus[(size_t)j*9]);
      store9(Vx2Vz1, &F.Vx2Vz1[(size_t)j*9]); store9(Vy2Vz1, &F.Vy2Vz1[(size_t)j*9]);
      store9(Vx2Vz2, &F.Vx2Vz2[(size_t)j*9]); store9(Vy2Vz2, &F.Vy2Vz2[(size_t)j*9]);
      store9(P1, &F.P2M1f[(size_t)j*9]); store9(P2, &F.P2M2f[(size_t)j*9]); store9(P3, &F.P2M3f[(size_t)j*9]);
      store9(Q1, &F.M2P1f[(size_t)j*9]); store9(Q2, &F.M2P2f[(size_t)j*9]); store9(Q3, &F.M2P3f[(size_t)j*9]);
    }
  }
}

/* -------- fault_init + fault_set (fault_info.cu:853-1074) --------------- */
void fault_set(oracle_solver *S, Fault &F, const cgfd_config *c, int id, int margin) {
  const size_t ns = S->siz_slice;
  auto z = [&](std::vector<real> &v) { v.assign(ns, 0); };
  z(F.T0x); z(F.T0y); z(F.T0z); z(F.mu_s); z(F.mu_d); z(F.Dc); z(F.C0);
  z(F.tTn); z(F.tTs1); z(F.tTs2);
  F.out.assign(11*ns, 0);
  F.united.assign(ns, 1); F.faultgrid.assign(ns, 0); F.rup_y.assign(ns, 0); F.rup_z.assign(ns, 0);
  F.flag_rup.assign(ns, 0); F.t0_flag.assign(ns, 0);
  for (int l = 0; l < 4; l++) F.fw[l].assign(18*ns, 0);
  F.T1x.assign(7*ns, 0); F.T1y.assign(7*ns, 0); F.T1z.assign(7*ns, 0);
  z(F.hT1x); z(F.hT1y); z(F.hT1z); z(F.mT1x); z(F.mT1y); z(F.mT1z);
  const size_t fsz = (size_t)S->nj*S->nk;
  for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++) {
    size_t pf = (size_t)j + (size_t)k*S->ny, src = id*fsz + (size_t)(j-3) + (size_t)(k-3)*S->nj;
    F.T0x[pf] = c->T0x[src]; F.T0y[pf] = c->T0y[src]; F.T0z[pf] = c->T0z[src];
    F.mu_s[pf] = c->mu_s[src]; F.mu_d[pf] = c->mu_d[src]; F.Dc[pf] = c->Dc[src]; F.C0[pf] = c->C0[src];
  }
  const int *fg = F.grid;
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) {
    size_t pf = (size_t)(j+S->nj1) + (size_t)(k+S->nk1)*S->ny;
    const real *vn = &F.vec_n[pf*3], *s1 = &F.vec_s1[pf*3], *s2 = &F.vec_s2[pf*3];
    F.o(CGFD_FAULT_TN)[pf]  = F.T0x[pf]*vn[0] + F.T0y[pf]*vn[1] + F.T0z[pf]*vn[2];
    F.o(CGFD_FAULT_TS1)[pf] = F.T0x[pf]*s1[0] + F.T0y[pf]*s1[1] + F.T0z[pf]*s1[2];
    F.o(CGFD_FAULT_TS2)[pf] = F.T0x[pf]*s2[0] + F.T0y[pf]*s2[1] + F.T0z[pf]*s2[2];
    int gj = j, gk = k;
    F.rup_y[pf] = (gj <= fg[0]+3 || gj >= fg[1]-3) ? 0 : 1;
    F.rup_z[pf] = (gk <= fg[2]+3 || gk >= fg[3]-3) ? 0 : 1;
    if (S->isfree)
      F.united[pf] = (gj >= margin && gj < S->nj - margin && gk >= margin) ? 0 : 1;
    else
      F.united[pf] = (gj >= margin && gj < S->nj - margin && gk >= margin && gk < S->nk - margin) ? 0 : 1;
    F.faultgrid[pf] = (gj >= fg[0]+3 && gj <= fg[1]-3 && gk >= fg[2]+3 && gk <= fg[3]-3) ? 1 : 0;
    F.o(CGFD_FAULT_INIT_T0)[pf] = (real)-9999.9;
    F.flag_rup[pf] = 0;
  }
}

/* ======================= per-stage kernels ============================== */

// wave2fault_gpu (transform.cu:101-212), united nodes
void wave2fault(oracle_solver *S, Fault &F, const real *w, const real *rhs, real *fc, real *frhs) {
  const size_t ic = S->siz_icmp, ns = S->siz_slice;
#pragma omp parallel for
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) {
    size_t pf = (size_t)(j+S->nj1) + (size_t)(k+S->nk1)*S->ny;
    if (F.united[pf] != 1) continue;
    size_t p = S->I(F.i0, j+S->nj1, k+S->nk1);
    real met[3][3] = { { S->M(1)[p], S->M(4)[p], S->M(7)[p] },
                       { S->M(2)[p], S->M(5)[p], S->M(8)[p] },
                       { S->M(3)[p], S->M(6)[p], S->M(9)[p] } };
    real jac = S->M(0)[p];
    real st[3][3] = { { w[TXX*ic+p], w[TXY*ic+p], w[TXZ*ic+p] },
                      { w[TXY*ic+p], w[TYY*ic+p], w[TYZ*ic+p] },
                      { w[TXZ*ic+p], w[TYZ*ic+p], w[TZZ*ic+p] } };
    real tr[3][3];
    mm3(st, met, tr);
    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) tr[a][b] *= jac;
    F.T1x[3*ns+pf] = tr[0][0]; F.T1y[3*ns+pf] = tr[1][0]; F.T1z[3*ns+pf] = tr[2][0];
    for (int m = 0; m < 2; m++) {
      real *f = fc + m*ns;
      f[FVX*2*ns+pf] = w[VX*ic+p]; f[FVY*2*ns+pf] = w[VY*ic+p]; f[FVZ*2*ns+pf] = w[VZ*ic+p];
      f[FT2X*2*ns+pf] = tr[0][1]; f[FT2Y*2*ns+pf] = tr[1][1]; f[FT2Z*2*ns+pf] = tr[2][1];
      f[FT3X*2*ns+pf] = tr[0][2]; f[FT3Y*2*ns+pf] = tr[1][2]; f[FT3Z*2*ns+pf] = tr[2][2];
    }
    real hs[3][3] = { { rhs[TXX*ic+p], rhs[TXY*ic+p], rhs[TXZ*ic+p] },
                      { rhs[TXY*ic+p], rhs[TYY*ic+p], rhs[TYZ*ic+p] },
                      { rhs[TXZ*ic+p], rhs[TYZ*ic+p], rhs[TZZ*ic+p] } };
    mm3(hs, met, tr);
    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) tr[a][b] *= jac;
    for (int m = 0; m < 2; m++) {
      real *f = frhs + m*ns;
      f[FT2X*2*ns+pf] = tr[0][1]; f[FT2Y*2*ns+pf] = tr[1][1]; f[FT2Z*2*ns+pf] = tr[2][1];
      f[FT3X*2*ns+pf] = tr[0][2]; f[FT3Y*2*ns+pf] = tr[1][2]; f[FT3Z*2*ns+pf] = tr[2][2];
    }
  }
}

// fault2wave_gpu (transform.cu:293-376), split nodes; keeps the Txz/Tyz swap
void fault2wave(oracle_solver *S, Fault &F, real *w, const real *fc) {
  const size_t ic = S->siz_icmp, ns = S->siz_slice;
#pragma omp parallel for
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) {
    size_t pf = (size_t)(j+S->nj1) + (size_t)(k+S->nk1)*S->ny;
    if (F.united[pf] != 0) continue;
    size_t p = S->I(F.i0, j+S->nj1, k+S->nk1);
    real met[3][3] = { { S->M(1)[p], S->M(4)[p], S->M(7)[p] },
                       { S->M(2)[p], S->M(5)[p], S->M(8)[p] },
                       { S->M(3)[p], S->M(6)[p], S->M(9)[p] } };
    real rj = 1.0/S->M(0)[p];
    real tr[3][3];
    tr[0][0] = F.T1x[3*ns+pf]; tr[1][0] = F.T1y[3*ns+pf]; tr[2][0] = F.T1z[3*ns+pf];
    auto avg = [&](int cmp) { return (fc[cmp*2*ns+pf] + fc[cmp*2*ns+pf+ns]) * (real)0.5; };
    tr[0][1] = avg(FT2X); tr[1][1] = avg(FT2Y); tr[2][1] = avg(FT2Z);
    tr[0][2] = avg(FT3X); tr[1][2] = avg(FT3Y); tr[2][2] = avg(FT3Z);
    inv3(met);
    real st[3][3];
    mm3(tr, met, st);
    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) st[a][b] *= rj;
    w[VX*ic+p] = avg(FVX); w[VY*ic+p] = avg(FVY); w[VZ*ic+p] = avg(FVZ);
    w[TXX*ic+p] = st[0][0]; w[TYY*ic+p] = st[1][1]; w[TZZ*ic+p] = st[2][2];
    w[TXY*ic+p] = (st[0][1] + st[1][0]) * (real)0.5;
    w[TYZ*ic+p] = (st[0][2] + st[2][0]) * (real)0.5;   // swapped as in the reference
    w[TXZ*ic+p] = (st[1][2] + st[2][1]) * (real)0.5;
  }
}

// trial_slipweakening_gpu (trial_slipweakening.cu:92-388)
void trial(oracle_solver *S, Fault &F, const real *w, real *fc, const real *fpre, int jdir, int kdir) {
  const size_t ic = S->siz_icmp, ns = S->siz_slice;
  const int ny = S->ny;
  const real dt = S->dt;
#pragma omp parallel for
  for (int iz = 0; iz < S->nk; iz++) for (int iy = 0; iy < S->nj; iy++) {
    size_t pf = (size_t)(iy+S->nj1) + (size_t)(iz+S->nk1)*ny;
    if (F.united[pf] != 0) continue;
    real Mrho[2], Rx[2], Ry[2], Rz[2];
    for (int m = 0; m < 2; m++) {
      size_t p = S->I(F.i0, iy+S->nj1, iz+S->nk1);
      real jac = S->M(0)[p];
      real rho = F.rho_f[pf + m*ns];
      Mrho[m] = 0.5*jac*rho;
      for (int l = 1; l <= 3; l++) {
        size_t q = S->I(F.i0+(2*m-1)*l, iy+S->nj1, iz+S->nk1);
        real xix = S->M(1)[q], xiy = S->M(2)[q], xiz = S->M(3)[q], J = S->M(0)[q];
        real T1x = J*(xix*w[TXX*ic+q] + xiy*w[TXY*ic+q] + xiz*w[TXZ*ic+q]);
        real T1y = J*(xix*w[TXY*ic+q] + xiy*w[TYY*ic+q] + xiz*w[TYZ*ic+q]);
        real T1z = J*(xix*w[TXZ*ic+q] + xiy*w[TYZ*ic+q] + xiz*w[TZZ*ic+q]);
        size_t t = (size_t)(3+(2*m-1)*l)*ns + pf;
        F.T1x[t] = T1x; F.T1y[t] = T1y; F.T1z[t] = T1z;
      }
      const real *f = fc + m*ns;
      const real *T2x = f + FT2X*2*ns + pf, *T2y = f + FT2Y*2*ns + pf, *T2z = f + FT2Z*2*ns + pf;
      const real *T3x = f + FT3X*2*ns + pf, *T3y = f + FT3Y*2*ns + pf, *T3z = f + FT3Z*2*ns + pf;
      real DyT2x, DyT2y, DyT2z, DzT3x, DzT3y, DzT3z;
      if (F.rup_y[pf] == 1) { DyT2x = mac22(T2x,1,jdir); DyT2y = mac22(T2y,1,jdir); DyT2z = mac22(T2z,1,jdir); }
      else { DyT2x = macdrp(T2x,1,jdir); DyT2y = macdrp(T2y,1,jdir); DyT2z = macdrp(T2z,1,jdir); }
      if (F.rup_z[pf] == 1) { DzT3x = mac22(T3x,ny,kdir); DzT3y = mac22(T3y,ny,kdir); DzT3z = mac22(T3z,ny,kdir); }
      else { DzT3x = macdrp(T3x,ny,kdir); DzT3y = macdrp(T3y,ny,kdir); DzT3z = macdrp(T3z,ny,kdir); }
      int km = S->nk - (iz+1);
      int n_free = km + 3;
      if (S->isfree == 1 && km <= 3) {
        real vx[7], vy[7], vz[7];
        for (int l = -3; l <= 3; l++) {
          vx[l+3] = T3x[(long)l*ny]; vy[l+3] = T3y[(long)l*ny]; vz[l+3] = T3z[(long)l*ny];
        }
        vx[n_free] = 0; vy[n_free] = 0; vz[n_free] = 0;
        for (int l = n_free+1; l < 7; l++) { vx[l] = -vx[2*n_free-l]; vy[l] = -vy[2*n_free-l]; vz[l] = -vz[2*n_free-l]; }
        DzT3x = vec_c(vx+3, kdir); DzT3y = vec_c(vy+3, kdir); DzT3z = vec_c(vz+3, kdir);
      }
      if (m == 0) {
        Rx[m] = (real)(A1*F.T1x[2*ns+pf] + A2*F.T1x[1*ns+pf] + A3*F.T1x[0*ns+pf]);
        Ry[m] = (real)(A1*F.T1y[2*ns+pf] + A2*F.T1y[1*ns+pf] + A3*F.T1y[0*ns+pf]);
        Rz[m] = (real)(A1*F.T1z[2*ns+pf] + A2*F.T1z[1*ns+pf] + A3*F.T1z[0*ns+pf]);
      } else {
        Rx[m] = (real)(A1*F.T1x[4*ns+pf] + A2*F.T1x[5*ns+pf] + A3*F.T1x[6*ns+pf]);
        Ry[m] = (real)(A1*F.T1y[4*ns+pf] + A2*F.T1y[5*ns+pf] + A3*F.T1y[6*ns+pf]);
        Rz[m] = (real)(A1*F.T1z[4*ns+pf] + A2*F.T1z[5*ns+pf] + A3*F.T1z[6*ns+pf]);
      }
      Rx[m] = 0.5*((2*m-1)*Rx[m] + (DyT2x + DzT3x));
      Ry[m] = 0.5*((2*m-1)*Ry[m] + (DyT2y + DzT3y));
      Rz[m] = 0.5*((2*m-1)*Rz[m] + (DyT2z + DzT3z));
    }
    real dVx = fpre[FVX*2*ns + pf + ns] - fpre[FVX*2*ns + pf];
    real dVy = fpre[FVY*2*ns + pf + ns] - fpre[FVY*2*ns + pf];
    real dVz = fpre[FVZ*2*ns + pf + ns] - fpre[FVZ*2*ns + pf];
    real Trial[3], Tl[3], Ts[3];
    Trial[0] = 2.0*(Mrho[0]*Mrho[1]*dVx/dt + Mrho[0]*Rx[1] - Mrho[1]*Rx[0])/(A0*(Mrho[0]+Mrho[1]));
    Trial[1] = 2.0*(Mrho[0]*Mrho[1]*dVy/dt + Mrho[0]*Ry[1] - Mrho[1]*Ry[0])/(A0*(Mrho[0]+Mrho[1]));
    Trial[2] = 2.0*(Mrho[0]*Mrho[1]*dVz/dt + Mrho[0]*Rz[1] - Mrho[1]*Rz[0])/(A0*(Mrho[0]+Mrho[1]));
    real s1[3] = { F.vec_s1[pf*3], F.vec_s1[pf*3+1], F.vec_s1[pf*3+2] };
    real s2[3] = { F.vec_s2[pf*3], F.vec_s2[pf*3+1], F.vec_s2[pf*3+2] };
    size_t p = S->I(F.i0, iy+S->nj1, iz+S->nk1);
    real vn[3] = { S->M(1)[p], S->M(2)[p], S->M(3)[p] };
    real vn0 = norm3(vn);
    real jacvec = S->M(0)[p] * vn0;
    for (int q = 0; q < 3; q++) vn[q] /= vn0;
    Tl[0] = Trial[0]/jacvec + F.T0x[pf];
    Tl[1] = Trial[1]/jacvec + F.T0y[pf];
    Tl[2] = Trial[2]/jacvec + F.T0z[pf];
    real Tn0 = dot3(Tl, vn);
    Ts[0] = Tl[0] - vn[0]*Tn0; Ts[1] = Tl[1] - vn[1]*Tn0; Ts[2] = Tl[2] - vn[2]*Tn0;
    real Ts0 = norm3(Ts);
    real Tau_n = Tn0, Tau_s = Ts0;
    int ifchange = 0;
    if (Tn0 >= 0.0) { Tau_n = 0.0; ifchange = 1; } else { Tau_n = Tn0; }
    real mu_s = F.mu_s[pf], mu_d = F.mu_d[pf], Slip = F.o(CGFD_FAULT_SLIP)[pf], Dc = F.Dc[pf], C0 = F.C0[pf];
    real fr;
    if (Slip <= Dc) fr = mu_s - (mu_s - mu_d) * Slip / Dc; else fr = mu_d;
    real Tau_c = -fr * Tau_n + C0;
    if (Ts0 >= Tau_c) { Tau_s = Tau_c; F.flag_rup[pf] = 1; ifchange = 1; }
    else { Tau_s = Ts0; F.flag_rup[pf] = 0; }
    real Tau[3];
    if (ifchange == 1) {
      if (std::fabs(Ts0) < 1e-1) {
        for (int q = 0; q < 3; q++) Tau[q] = Tau_n * vn[q];
      } else {
        for (int q = 0; q < 3; q++) Tau[q] = Tau_n * vn[q] + (Tau_s/Ts0) * Ts[q];
      }
    } else {
      for (int q = 0; q < 3; q++) Tau[q] = Tl[q];
    }
    if (ifchange == 1) {
      F.T1x[pf+3*ns] = (Tau[0] - F.T0x[pf])*jacvec;
      F.T1y[pf+3*ns] = (Tau[1] - F.T0y[pf])*jacvec;
      F.T1z[pf+3*ns] = (Tau[2] - F.T0z[pf])*jacvec;
    } else {
      F.T1x[pf+3*ns] = Trial[0]; F.T1y[pf+3*ns] = Trial[1]; F.T1z[pf+3*ns] = Trial[2];
    }
    F.tTs1[pf] = dot3(Tau, s1);
    F.tTs2[pf] = dot3(Tau, s2);
    F.tTn[pf] = Tau_n;
  }
}

// conservative traction J*(e . sigma) of stress components at point q
inline void tract(const real *w, size_t ic, size_t q, real ex, real ey, real ez, real J,
                  real &tx, real &ty, real &tz) {
  tx = J*(ex*w[TXX*ic+q] + ey*w[TXY*ic+q] + ez*w[TXZ*ic+q]);
  ty = J*(ex*w[TXY*ic+q] + ey*w[TYY*ic+q] + ez*w[TYZ*ic+q]);
  tz = J*(ex*w[TXZ*ic+q] + ey*w[TYZ*ic+q] + ez*w[TZZ*ic+q]);
}

/* volume RHS: sv_curv_col_el_iso_rhs_inner_gpu (sv_curv_col_el_iso_gpu.cu:232-388) */
void rhs_inner(oracle_solver *S, const real *w, real *h, int idir, int jdir, int kdir) {
  const size_t ic = S->siz_icmp;
  long shx[5], shy[5], shz[5];
  real cx[5], cy[5], cz[5];
  for (int n = 0; n < 5; n++) {
    shx[n] = OP_IDX[idir][n]; shy[n] = OP_IDX[jdir][n]*(long)S->siz_iy; shz[n] = OP_IDX[kdir][n]*(long)S->siz_iz;
    cx[n] = OP_COEF[idir][n]; cy[n] = OP_COEF[jdir][n]; cz[n] = OP_COEF[kdir][n];
  }
  auto D = [&](const real *f, const long *sh, const real *cf) {
    return cf[0]*f[sh[0]] + cf[1]*f[sh[1]] + cf[2]*f[sh[2]] + cf[3]*f[sh[3]] + cf[4]*f[sh[4]];
  };
#pragma omp parallel for collapse(2)
  for (int k = S->nk1; k <= S->nk2; k++) for (int j = S->nj1; j <= S->nj2; j++)
    for (int i = S->ni1; i <= S->ni2; i++) {
      size_t p = S->I(i,j,k);
      const real *Vx = w + VX*ic + p, *Vy = w + VY*ic + p, *Vz = w + VZ*ic + p;
      const real *Txx = w + TXX*ic + p, *Tyy = w + TYY*ic + p, *Tzz = w + TZZ*ic + p;
      const real *Txz = w + TXZ*ic + p, *Tyz = w + TYZ*ic + p, *Txy = w + TXY*ic + p;
      real DxVx = D(Vx,shx,cx), DyVx = D(Vx,shy,cy), DzVx = D(Vx,shz,cz);
      real DxVy = D(Vy,shx,cx), DyVy = D(Vy,shy,cy), DzVy = D(Vy,shz,cz);
      real DxVz = D(Vz,shx,cx), DyVz = D(Vz,shy,cy), DzVz = D(Vz,shz,cz);
      real DxTxx = D(Txx,shx,cx), DyTxx = D(Txx,shy,cy), DzTxx = D(Txx,shz,cz);
      real DxTyy = D(Tyy,shx,cx), DyTyy = D(Tyy,shy,cy), DzTyy = D(Tyy,shz,cz);
      real DxTzz = D(Tzz,shx,cx), DyTzz = D(Tzz,shy,cy), DzTzz = D(Tzz,shz,cz);
      real DxTxz = D(Txz,shx,cx), DyTxz = D(Txz,shy,cy), DzTxz = D(Txz,shz,cz);
      real DxTyz = D(Tyz,shx,cx), DyTyz = D(Tyz,shy,cy), DzTyz = D(Tyz,shz,cz);
      real DxTxy = D(Txy,shx,cx), DyTxy = D(Txy,shy,cy), DzTxy = D(Txy,shz,cz);
      real xix = S->M(1)[p], xiy = S->M(2)[p], xiz = S->M(3)[p];
      real etx = S->M(4)[p], ety = S->M(5)[p], etz = S->M(6)[p];
      real ztx = S->M(7)[p], zty = S->M(8)[p], ztz = S->M(9)[p];
      real lam = S->lam[p], mu = S->mu[p], slw = S->rho[p];
      real lam2mu = lam + 2.0*mu;
      h[VX*ic+p] = slw*( xix*DxTxx + xiy*DxTxy + xiz*DxTxz + etx*DyTxx + ety*DyTxy + etz*DyTxz
                        + ztx*DzTxx + zty*DzTxy + ztz*DzTxz );
      h[VY*ic+p] = slw*( xix*DxTxy + xiy*DxTyy + xiz*DxTyz + etx*DyTxy + ety*DyTyy + etz*DyTyz
                        + ztx*DzTxy + zty*DzTyy + ztz*DzTyz );
      h[VZ*ic+p] = slw*( xix*DxTxz + xiy*DxTyz + xiz*DxTzz + etx*DyTxz + ety*DyTyz + etz*DyTzz
                        + ztx*DzTxz + zty*DzTyz + ztz*DzTzz );
      h[TXX*ic+p] = lam2mu*(xix*DxVx + etx*DyVx + ztx*DzVx)
                  + lam*(xiy*DxVy + ety*DyVy + zty*DzVy + xiz*DxVz + etz*DyVz + ztz*DzVz);
      h[TYY*ic+p] = lam2mu*(xiy*DxVy + ety*DyVy + zty*DzVy)
                  + lam*(xix*DxVx + etx*DyVx + ztx*DzVx + xiz*DxVz + etz*DyVz + ztz*DzVz);
      h[TZZ*ic+p] = lam2mu*(xiz*DxVz + etz*DyVz + ztz*DzVz)
                  + lam*(xix*DxVx + etx*DyVx + ztx*DzVx + xiy*DxVy + ety*DyVy + zty*DzVy);
      h[TXY*ic+p] = mu*(xiy*DxVx + xix*DxVy + ety*DyVx + etx*DyVy + zty*DzVx + ztx*DzVy);
      h[TXZ*ic+p] = mu*(xiz*DxVx + xix*DxVz + etz*DyVx + etx*DyVz + ztz*DzVx + ztx*DzVz);
      h[TYZ*ic+p] = mu*(xiz*DxVy + xiy*DxVz + etz*DyVy + ety*DyVz + ztz*DzVy + zty*DzVz);
    }
}

/* traction image: sv_curv_col_el_iso_rhs_timg_z2_gpu (:399-600) */
void rhs_timg(oracle_solver *S, const real *w, real *h, int idir, int jdir, int kdir) {
  const size_t ic = S->siz_icmp;
  const int *fx = OP_IDX[idir], *fy = OP_IDX[jdir], *fz = OP_IDX[kdir];
  const int k_min = S->nk2 - fz[4];
  const real *jac = S->M(0);
  // rows: the stress components forming the traction for hVx, hVy, hVz
  const int rows[3][3] = { {TXX, TXY, TXZ}, {TXY, TYY, TYZ}, {TXZ, TYZ, TZZ} };
  for (int k = k_min; k <= S->nk2; k++) {
    int n_free = S->nk2 - k - fz[0];
#pragma omp parallel for
    for (int j = S->nj1; j <= S->nj2; j++) for (int i = S->ni1; i <= S->ni2; i++) {
      size_t p = S->I(i,j,k);
      real slwjac = S->rho[p] / jac[p];
      for (int r = 0; r < 3; r++) {
        const real *A = w + rows[r][0]*ic, *B = w + rows[r][1]*ic, *C = w + rows[r][2]*ic;
        real vxi[5], vet[5], vzt[5];
        for (int n = 0; n < 5; n++) {
          size_t q = p + fx[n];
          vxi[n] = jac[q]*(S->M(1)[q]*A[q] + S->M(2)[q]*B[q] + S->M(3)[q]*C[q]);
        }
        for (int n = 0; n < 5; n++) {
          size_t q = p + (long)fy[n]*S->siz_iy;
          vet[n] = jac[q]*(S->M(4)[q]*A[q] + S->M(5)[q]*B[q] + S->M(6)[q]*C[q]);
        }
        int n;
        for (n = 0; n < n_free; n++) {
          size_t q = p + (long)fz[n]*S->siz_iz;
          vzt[n] = jac[q]*(S->M(7)[q]*A[q] + S->M(8)[q]*B[q] + S->M(9)[q]*C[q]);
        }
        vzt[n_free] = 0.0;
        for (n = n_free+1; n < 5; n++) {
          int n_img = fz[n] - 2*(n - n_free);
          size_t q = p + (long)n_img*S->siz_iz;
          vzt[n] = -jac[q]*(S->M(7)[q]*A[q] + S->M(8)[q]*B[q] + S->M(9)[q]*C[q]);
        }
        real DxT = vec_drp(vxi, idir), DyT = vec_drp(vet, jdir), DzT = vec_drp(vzt, kdir);
        h[(VX+r)*ic+p] = (DxT + DyT + DzT) * slwjac;
      }
    }
  }
}

/* velocity below the surface: sv_curv_col_el_iso_rhs_vlow_z2_gpu (:607-747) */
void rhs_vlow(oracle_solver *S, const real *w, real *h, int idir, int jdir, int kdir) {
  const size_t ic = S->siz_icmp;
  for (int n = 0; n < 3; n++) {
    int k = S->nk2 - n;
#pragma omp parallel for
    for (int j = S->nj1; j <= S->nj2; j++) for (int i = S->ni1; i <= S->ni2; i++) {
      size_t p = S->I(i,j,k);
      real xix = S->M(1)[p], xiy = S->M(2)[p], xiz = S->M(3)[p];
      real etx = S->M(4)[p], ety = S->M(5)[p], etz = S->M(6)[p];
      real ztx = S->M(7)[p], zty = S->M(8)[p], ztz = S->M(9)[p];
      real lam = S->lam[p], mu = S->mu[p];
      real lam2mu = lam + 2.0*mu;
      const real *Vx = w + VX*ic + p, *Vy = w + VY*ic + p, *Vz = w + VZ*ic + p;
      long sy = (long)S->siz_iy, sz = (long)S->siz_iz;
      real DxVx = macdrp(Vx,1,idir), DyVx = macdrp(Vx,sy,jdir);
      real DxVy = macdrp(Vy,1,idir), DyVy = macdrp(Vy,sy,jdir);
      real DxVz = macdrp(Vz,1,idir), DyVz = macdrp(Vz,sy,jdir);
      real DzVx = 0, DzVy = 0, DzVz = 0;
      if (k == S->nk2) {
        size_t ij = ((size_t)i + (size_t)j*S->siz_iy)*9;
        const real *X = &S->matVx2Vz[ij], *Y = &S->matVy2Vz[ij];
        DzVx = X[0]*DxVx + X[1]*DxVy + X[2]*DxVz + Y[0]*DyVx + Y[1]*DyVy + Y[2]*DyVz;
        DzVy = X[3]*DxVx + X[4]*DxVy + X[5]*DxVz + Y[3]*DyVx + Y[4]*DyVy + Y[5]*DyVz;
        DzVz = X[6]*DxVx + X[7]*DxVy + X[8]*DxVz + Y[6]*DyVx + Y[7]*DyVy + Y[8]*DyVz;
      }
      if (k == S->nk2-1) { DzVx = mac22(Vx,sz,kdir); DzVy = mac22(Vy,sz,kdir); DzVz = mac22(Vz,sz,kdir); }
      if (k == S->nk2-2) { DzVx = mac24(Vx,sz,kdir); DzVy = mac24(Vy,sz,kdir); DzVz = mac24(Vz,sz,kdir); }
      h[TXX*ic+p] = lam2mu*(xix*DxVx + etx*DyVx + ztx*DzVx)
                  + lam*(xiy*DxVy + ety*DyVy + zty*DzVy + xiz*DxVz + etz*DyVz + ztz*DzVz);
      h[TYY*ic+p] = lam2mu*(xiy*DxVy + ety*DyVy + zty*DzVy)
                  + lam*(xix*DxVx + etx*DyVx + ztx*DzVx + xiz*DxVz + etz*DyVz + ztz*DzVz);
      h[TZZ*ic+p] = lam2mu*(xiz*DxVz + etz*DyVz + ztz*DzVz)
                  + lam*(xix*DxVx + etx*DyVx + ztx*DzVx + xiy*DxVy + ety*DyVy + zty*DzVy);
      h[TXY*ic+p] = mu*(xiy*DxVx + xix*DxVy + ety*DyVx + etx*DyVy + zty*DzVx + ztx*DzVy);
      h[TXZ*ic+p] = mu*(xiz*DxVx + xix*DxVz + etz*DyVx + etx*DyVz + ztz*DzVx + ztx*DzVz);
      h[TYZ*ic+p] = mu*(xiz*DxVy + xiy*DxVz + etz*DyVy + ety*DyVz + ztz*DzVy + zty*DzVz);
    }
  }
}

/* CFS-PML: sv_curv_col_el_iso_rhs_cfspml_gpu (:825-1290), faces in order */
void rhs_pml(oracle_solver *S, const real *w, real *h, int idir, int jdir, int kdir) {
  const size_t ic = S->siz_icmp;
  const int dirs[3] = { idir, jdir, kdir };
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
    PmlFace &F = S->pml[d][s];
    if (!F.on) continue;
    const int dr = dirs[d];
    long sh[5]; real cf[5];
    long stride = d == 0 ? 1 : (d == 1 ? (long)S->siz_iy : (long)S->siz_iz);
    for (int n = 0; n < 5; n++) { sh[n] = OP_IDX[dr][n]*stride; cf[n] = OP_COEF[dr][n]; }
    const real *pc = F.aux[F.cur].data();      // stage input level
    real *ph = F.aux[F.lvl[LRHS]].data();
    const int mc = 1 + 3*d;   // metric row of this direction
#pragma omp parallel for collapse(2)
    for (int iz = 0; iz < F.nk; iz++) for (int iy = 0; iy < F.nj; iy++) for (int ix = 0; ix < F.ni; ix++) {
      size_t pa = (size_t)iz*F.nj*F.ni + (size_t)iy*F.ni + ix;
      size_t p = S->I(ix+F.i1, iy+F.j1, iz+F.k1);
      int layer = d == 0 ? ix : (d == 1 ? iy : iz);
      real cD = F.D[layer], cA = F.A[layer], cB = F.B[layer];
      real cB1 = cB - 1.0;
      real ex = S->M(mc)[p], ey = S->M(mc+1)[p], ez = S->M(mc+2)[p];
      real lam = S->lam[p], mu = S->mu[p], slw = S->rho[p];
      real lam2mu = lam + 2.0*mu;
      real Dv[9];
      for (int c = 0; c < 9; c++) {
        const real *f = w + c*ic + p;
        Dv[c] = cf[0]*f[sh[0]] + cf[1]*f[sh[1]] + cf[2]*f[sh[2]] + cf[3]*f[sh[3]] + cf[4]*f[sh[4]];
      }
      real r[9];
      r[VX] = slw*(ex*Dv[TXX] + ey*Dv[TXY] + ez*Dv[TXZ]);
      r[VY] = slw*(ex*Dv[TXY] + ey*Dv[TYY] + ez*Dv[TYZ]);
      r[VZ] = slw*(ex*Dv[TXZ] + ey*Dv[TYZ] + ez*Dv[TZZ]);
      r[TXX] = lam2mu*ex*Dv[VX] + lam*ey*Dv[VY] + lam*ez*Dv[VZ];
      r[TYY] = lam*ex*Dv[VX] + lam2mu*ey*Dv[VY] + lam*ez*Dv[VZ];
      r[TZZ] = lam*ex*Dv[VX] + lam*ey*Dv[VY] + lam2mu*ez*Dv[VZ];
      r[TXY] = mu*(ey*Dv[VX] + ex*Dv[VY]);
      r[TXZ] = mu*(ez*Dv[VX] + ex*Dv[VZ]);
      r[TYZ] = mu*(ez*Dv[VY] + ey*Dv[VZ]);
      for (int c = 0; c < 9; c++) {
        h[c*ic+p] += cB1*r[c] - cB*pc[c*F.siz+pa];
        ph[c*F.siz+pa] = cD*r[c] - cA*pc[c*F.siz+pa];
      }
      if (d < 2 && S->isfree == 1 && (iz+F.k1) == S->nk2) {
        size_t ij = ((size_t)(ix+F.i1) + (size_t)(iy+F.j1)*S->siz_iy)*9;
        const real *X = d == 0 ? &S->matVx2Vz[ij] : &S->matVy2Vz[ij];
        real DzVx = X[0]*Dv[VX] + X[1]*Dv[VY] + X[2]*Dv[VZ];
        real DzVy = X[3]*Dv[VX] + X[4]*Dv[VY] + X[5]*Dv[VZ];
        real DzVz = X[6]*Dv[VX] + X[7]*Dv[VY] + X[8]*Dv[VZ];
        real ztx = S->M(7)[p], zty = S->M(8)[p], ztz = S->M(9)[p];
        real q[9];
        q[TXX] = lam2mu*(ztx*DzVx) + lam*(zty*DzVy + ztz*DzVz);
        q[TYY] = lam2mu*(zty*DzVy) + lam*(ztx*DzVx + ztz*DzVz);
        q[TZZ] = lam2mu*(ztz*DzVz) + lam*(ztx*DzVx + zty*DzVy);
        q[TXY] = mu*(zty*DzVx + ztx*DzVy);
        q[TXZ] = mu*(ztz*DzVx + ztx*DzVz);
        q[TYZ] = mu*(ztz*DzVy + zty*DzVz);
        for (int c = TXX; c <= TXY; c++) {
          h[c*ic+p] += (cB - 1.0) * q[c];
          ph[c*F.siz+pa] += cD * q[c];
        }
      }
    }
  }
}

/* fault velocity RHS: sv_curv_col_el_iso_rhs_fault_velo_gpu
 * (sv_curv_col_el_iso_fault_gpu.cu:192-429) */
void rhs_fault_velo(oracle_solver *S, Fault &F, const real *w, real *h, const real *fc, real *frhs,
                    int idir, int jdir, int kdir) {
  const size_t ic = S->siz_icmp, ns = S->siz_slice;
  const int ny = S->ny;
#pragma omp parallel for
  for (int iz = 0; iz < S->nk; iz++) for (int iy = 0; iy < S->nj; iy++) {
    size_t pf = (size_t)(iy+S->nj1) + (size_t)(iz+S->nk1)*ny;
    if (F.united[pf] != 0) continue;
    int km = S->nk - (iz+1), n_free = km + 3;
    const int jj = iy+S->nj1, kk = iz+S->nk1;
    for (int i = F.i0-3; i <= F.i0+3; i++) {
      int n = F.i0 - i;
      if (n == 0) continue;
      real v1x[7], v1y[7], v1z[7], v2x[7], v2y[7], v2z[7], v3x[7], v3y[7], v3z[7];
      for (int l = -3; l <= 3; l++) {
        size_t q = S->I(i+l, jj, kk);
        tract(w, ic, q, S->M(1)[q], S->M(2)[q], S->M(3)[q], S->M(0)[q], v1x[l+3], v1y[l+3], v1z[l+3]);
        q = S->I(i, jj+l, kk);
        tract(w, ic, q, S->M(4)[q], S->M(5)[q], S->M(6)[q], S->M(0)[q], v2x[l+3], v2y[l+3], v2z[l+3]);
        q = S->I(i, jj, kk+l);
        tract(w, ic, q, S->M(7)[q], S->M(8)[q], S->M(9)[q], S->M(0)[q], v3x[l+3], v3y[l+3], v3z[l+3]);
      }
      v1x[n+3] = F.T1x[3*ns+pf]; v1y[n+3] = F.T1y[3*ns+pf]; v1z[n+3] = F.T1z[3*ns+pf];
      real *V[3] = { v1x, v1y, v1z };
      for (int c = 0; c < 3; c++) {
        real *v = V[c];
        if (n == 2) { v[6] = 2.0*v[5] - v[4]; }
        if (n == 1) { v[5] = 2.0*v[4] - v[3]; v[6] = 2.0*v[4] - v[2]; }
        if (n == -1) { v[0] = 2.0*v[2] - v[4]; v[1] = 2.0*v[2] - v[3]; }
        if (n == -2) { v[0] = 2.0*v[1] - v[2]; }
      }
      if (S->isfree == 1 && km <= 3) {
        real *Z[3] = { v3x, v3y, v3z };
        for (int c = 0; c < 3; c++) {
          Z[c][n_free] = 0.0;
          for (int l = n_free+1; l < 7; l++) Z[c][l] = -Z[c][2*n_free-l];
        }
      }
      real DxT1x = vec_c(v1x+3, idir), DxT1y = vec_c(v1y+3, idir), DxT1z = vec_c(v1z+3, idir);
      real DyT2x = vec_c(v2x+3, jdir), DyT2y = vec_c(v2y+3, jdir), DyT2z = vec_c(v2z+3, jdir);
      real DzT3x = vec_c(v3x+3, kdir), DzT3y = vec_c(v3y+3, kdir), DzT3z = vec_c(v3z+3, kdir);
      size_t p = S->I(i, jj, kk);
      real rr = S->rho[p] / S->M(0)[p];
      h[VX*ic+p] = (DxT1x + DyT2x + DzT3x)*rr;
      h[VY*ic+p] = (DxT1y + DyT2y + DzT3y)*rr;
      h[VZ*ic+p] = (DxT1z + DyT2z + DzT3z)*rr;
    }
    for (int m = 0; m < 2; m++) {
      real DxT1x, DxT1y, DxT1z;
      const real *T1[3] = { F.T1x.data(), F.T1y.data(), F.T1z.data() };
      real Dx[3];
      for (int c = 0; c < 3; c++) {
        const real *t = T1[c];
        if (m == 0)
          Dx[c] = (real)(A0*t[pf+3*ns] - A1*t[pf+2*ns] - A2*t[pf+1*ns] - A3*t[pf+0*ns]);
        else
          Dx[c] = (real)(-A0*t[pf+3*ns] + A1*t[pf+4*ns] + A2*t[pf+5*ns] + A3*t[pf+6*ns]);
      }
      DxT1x = Dx[0]; DxT1y = Dx[1]; DxT1z = Dx[2];
      const real *f = fc + m*ns;
      const real *T2x = f + FT2X*2*ns + pf, *T2y = f + FT2Y*2*ns + pf, *T2z = f + FT2Z*2*ns + pf;
      const real *T3x = f + FT3X*2*ns + pf, *T3y = f + FT3Y*2*ns + pf, *T3z = f + FT3Z*2*ns + pf;
      real DyT2x, DyT2y, DyT2z, DzT3x, DzT3y, DzT3z;
      if (F.rup_y[pf] == 1) { DyT2x = mac22(T2x,1,jdir); DyT2y = mac22(T2y,1,jdir); DyT2z = mac22(T2z,1,jdir); }
      else { DyT2x = macdrp(T2x,1,jdir); DyT2y = macdrp(T2y,1,jdir); DyT2z = macdrp(T2z,1,jdir); }
      if (F.rup_z[pf] == 1) { DzT3x = mac22(T3x,ny,kdir); DzT3y = mac22(T3y,ny,kdir); DzT3z = mac22(T3z,ny,kdir); }
      else { DzT3x = macdrp(T3x,ny,kdir); DzT3y = macdrp(T3y,ny,kdir); DzT3z = macdrp(T3z,ny,kdir); }
      if (S->isfree == 1 && km <= 3) {
        real vx[7], vy[7], vz[7];
        for (int l = -3; l <= 3; l++) { vx[l+3] = T3x[(long)l*ny]; vy[l+3] = T3y[(long)l*ny]; vz[l+3] = T3z[(long)l*ny]; }
        vx[n_free] = 0; vy[n_free] = 0; vz[n_free] = 0;
        for (int l = n_free+1; l < 7; l++) { vx[l] = -vx[2*n_free-l]; vy[l] = -vy[2*n_free-l]; vz[l] = -vz[2*n_free-l]; }
        DzT3x = vec_c(vx+3, kdir); DzT3y = vec_c(vy+3, kdir); DzT3z = vec_c(vz+3, kdir);
      }
      size_t p = S->I(F.i0, jj, kk);
      real rr = 1.0 / (F.rho_f[pf + m*ns] * S->M(0)[p]);
      real *fh = frhs + m*ns;
      fh[FVX*2*ns+pf] = (DxT1x + DyT2x + DzT3x)*rr;
      fh[FVY*2*ns+pf] = (DxT1y + DyT2y + DzT3y)*rr;
      fh[FVZ*2*ns+pf] = (DxT1z + DyT2z + DzT3z)*rr;
    }
  }
}

/* fault stress RHS: sv_curv_col_el_iso_rhs_fault_stress_F_gpu (:432-1159)
 * and _B_gpu (:1162-1879); idir selects the variant */
void rhs_fault_stress(oracle_solver *S, Fault &F, const real *w, real *h, const real *fc, real *frhs,
                      int idir, int jdir, int kdir) {
  const size_t ic = S->siz_icmp, ns = S->siz_slice;
  const int ny = S->ny;
  const long sy = (long)S->siz_iy, sz = (long)S->siz_iz;
#pragma omp parallel for
  for (int iz = 0; iz < S->nk; iz++) for (int iy = 0; iy < S->nj; iy++) {
    size_t pf = (size_t)(iy+S->nj1) + (size_t)(iz+S->nk1)*ny;
    if (F.united[pf] != 0) continue;
    const int km = S->nk - (iz+1);
    const int jj = iy+S->nj1, kk = iz+S->nk1;
    const int i0 = F.i0;
    const real *Vx = w + VX*ic, *Vy = w + VY*ic, *Vz = w + VZ*ic;
    const real *fVx = fc + FVX*2*ns, *fVy = fc + FVY*2*ns, *fVz = fc + FVZ*2*ns;
    real DxVx[8], DxVy[8], DxVz[8], DyVx[8], DyVy[8], DyVz[8], DzVx[8], DzVy[8], DzVz[8];
    for (int q = 0; q < 8; q++) { DxVx[q]=DxVy[q]=DxVz[q]=DyVx[q]=DyVy[q]=DyVz[q]=DzVx[q]=DzVy[q]=DzVz[q]=0; }
    auto P = [&](int i) { return S->I(i, jj, kk); };
    if (idir == 1) {
      // A, B, C on the plus side, forward operators
      size_t p = P(i0+3);
      DxVx[7] = macdrp(Vx+p,1,1); DxVy[7] = macdrp(Vy+p,1,1); DxVz[7] = macdrp(Vz+p,1,1);
      p = P(i0+2);
      DxVx[6] = mac24(Vx+p,1,1); DxVy[6] = mac24(Vy+p,1,1); DxVz[6] = mac24(Vz+p,1,1);
      p = P(i0+1);
      DxVx[5] = mac22(Vx+p,1,1); DxVy[5] = mac22(Vy+p,1,1); DxVz[5] = mac22(Vz+p,1,1);
    } else {
      size_t p = P(i0-3);
      DxVx[0] = macdrp(Vx+p,1,0); DxVy[0] = macdrp(Vy+p,1,0); DxVz[0] = macdrp(Vz+p,1,0);
      p = P(i0-2);
      DxVx[1] = mac24(Vx+p,1,0); DxVy[1] = mac24(Vy+p,1,0); DxVz[1] = mac24(Vz+p,1,0);
      p = P(i0-1);
      DxVx[2] = mac22(Vx+p,1,0); DxVy[2] = mac22(Vy+p,1,0); DxVz[2] = mac22(Vz+p,1,0);
    }
    // split nodes D- (3) and D+ (4): along-fault derivatives
    for (int m = 0; m < 2; m++) {
      const real *ax = fVx + pf + m*ns, *ay = fVy + pf + m*ns, *az = fVz + pf + m*ns;
      int q = 3 + m;
      if (F.rup_y[pf] == 1) { DyVx[q] = mac22(ax,1,jdir); DyVy[q] = mac22(ay,1,jdir); DyVz[q] = mac22(az,1,jdir); }
      else { DyVx[q] = macdrp(ax,1,jdir); DyVy[q] = macdrp(ay,1,jdir); DyVz[q] = macdrp(az,1,jdir); }
      if (F.rup_z[pf] == 1) { DzVx[q] = mac22(ax,ny,kdir); DzVy[q] = mac22(ay,ny,kdir); DzVz[q] = mac22(az,ny,kdir); }
      else { DzVx[q] = macdrp(ax,ny,kdir); DzVy[q] = macdrp(ay,ny,kdir); DzVz[q] = macdrp(az,ny,kdir); }
    }
    const size_t ix9 = pf*9;
    real dtT1[3];
    auto get_dtT1 = [&]() {
      if (F.faultgrid[pf] == 1) { dtT1[0] = F.hT1x[pf]; dtT1[1] = F.hT1y[pf]; dtT1[2] = F.hT1z[pf]; }
      else { dtT1[0] = 0.0; dtT1[1] = 0.0; dtT1[2] = 0.0; }
    };
    real o1[3], o2[3], o3[3], o4[3], o5[3], m1[3][3], m2[3][3], m3[3][3], m4[3][3], m5[3][3];
    auto split_general = [&]() {
      if (S->imethod == 1) {
        real dxV[3], dyV1[3] = { DyVx[3], DyVy[3], DyVz[3] }, dzV1[3] = { DzVx[3], DzVy[3], DzVz[3] };
        real dyV2[3] = { DyVx[4], DyVy[4], DyVz[4] }, dzV2[3] = { DzVx[4], DzVy[4], DzVz[4] };
        if (idir == 1) {
          size_t p = P(i0+1);
          DxVx[4] = (Vx[p] - fVx[pf+ns]); DxVy[4] = (Vy[p] - fVy[pf+ns]); DxVz[4] = (Vz[p] - fVz[pf+ns]);
          dxV[0] = DxVx[4]; dxV[1] = DxVy[4]; dxV[2] = DxVz[4];
          load9(&F.P2M1[ix9], m1); load9(&F.P2M2[ix9], m2); load9(&F.P2M3[ix9], m3);
          load9(&F.P2M4[ix9], m4); load9(&F.P2M5[ix9], m5);
          mv3(m1, dxV, o1); mv3(m2, dyV2, o2); mv3(m3, dzV2, o3); mv3(m4, dyV1, o4); mv3(m5, dzV1, o5);
          DxVx[3] = o1[0] + o2[0] + o3[0] - o4[0] - o5[0];
          DxVy[3] = o1[1] + o2[1] + o3[1] - o4[1] - o5[1];
          DxVz[3] = o1[2] + o2[2] + o3[2] - o4[2] - o5[2];
        } else {
          size_t p = P(i0-1);
          DxVx[3] = (fVx[pf] - Vx[p]); DxVy[3] = (fVy[pf] - Vy[p]); DxVz[3] = (fVz[pf] - Vz[p]);
          dxV[0] = DxVx[3]; dxV[1] = DxVy[3]; dxV[2] = DxVz[3];
          load9(&F.M2P1[ix9], m1); load9(&F.M2P2[ix9], m2); load9(&F.M2P3[ix9], m3);
          load9(&F.M2P4[ix9], m4); load9(&F.M2P5[ix9], m5);
          mv3(m1, dxV, o1); mv3(m2, dyV1, o2); mv3(m3, dzV1, o3); mv3(m4, dyV2, o4); mv3(m5, dzV2, o5);
          DxVx[4] = o1[0] + o2[0] + o3[0] - o4[0] - o5[0];
          DxVy[4] = o1[1] + o2[1] + o3[1] - o4[1] - o5[1];
          DxVz[4] = o1[2] + o2[2] + o3[2] - o4[2] - o5[2];
        }
      } else if (S->imethod == 2) {
        get_dtT1();
        real dy[3], dzz[3];
        // plus
        dy[0] = DyVx[4]; dy[1] = DyVy[4]; dy[2] = DyVz[4]; dzz[0] = DzVx[4]; dzz[1] = DzVy[4]; dzz[2] = DzVz[4];
        load9(&F.T1toVxPlus[ix9], m1); load9(&F.VytoVxPlus[ix9], m2); load9(&F.VztoVxPlus[ix9], m3);
        mv3(m1, dtT1, o1); mv3(m2, dy, o2); mv3(m3, dzz, o3);
        real px = o1[0] - o2[0] - o3[0], py = o1[1] - o2[1] - o3[1], pz = o1[2] - o2[2] - o3[2];
        // minus
        dy[0] = DyVx[3]; dy[1] = DyVy[3]; dy[2] = DyVz[3]; dzz[0] = DzVx[3]; dzz[1] = DzVy[3]; dzz[2] = DzVz[3];
        load9(&F.T1toVxMin[ix9], m1); load9(&F.VytoVxMin[ix9], m2); load9(&F.VztoVxMin[ix9], m3);
        mv3(m1, dtT1, o1); mv3(m2, dy, o2); mv3(m3, dzz, o3);
        DxVx[3] = o1[0] - o2[0] - o3[0]; DxVy[3] = o1[1] - o2[1] - o3[1]; DxVz[3] = o1[2] - o2[2] - o3[2];
        DxVx[4] = px; DxVy[4] = py; DxVz[4] = pz;
      }
    };
    split_general();
    if (S->isfree == 1 && km == 0) {
      const size_t jr = (size_t)(iy+3)*9;
      real dyV1[3] = { DyVx[3], DyVy[3], DyVz[3] }, dyV2[3] = { DyVx[4], DyVy[4], DyVz[4] };
      if (S->imethod == 1) {
        if (idir == 1) {
          real dxV2[3] = { DxVx[4], DxVy[4], DxVz[4] };
          load9(&F.P2M1f[jr], m1); load9(&F.P2M2f[jr], m2); load9(&F.P2M3f[jr], m3);
          mv3(m1, dxV2, o1); mv3(m2, dyV2, o2); mv3(m3, dyV1, o3);
          DxVx[3] = o1[0] + o2[0] - o3[0]; DxVy[3] = o1[1] + o2[1] - o3[1]; DxVz[3] = o1[2] + o2[2] - o3[2];
        } else {
          real dxV1[3] = { DxVx[3], DxVy[3], DxVz[3] };
          load9(&F.M2P1f[jr], m1); load9(&F.M2P2f[jr], m2); load9(&F.M2P3f[jr], m3);
          mv3(m1, dxV1, o1); mv3(m2, dyV1, o2); mv3(m3, dyV2, o3);
          DxVx[4] = o1[0] + o2[0] - o3[0]; DxVy[4] = o1[1] + o2[1] - o3[1]; DxVz[4] = o1[2] + o2[2] - o3[2];
        }
      }
      if (S->imethod == 2) {
        get_dtT1();
        load9(&F.T1toVxfPlus[jr], m1); load9(&F.VytoVxfPlus[jr], m2);
        mv3(m1, dtT1, o1); mv3(m2, dyV2, o2);
        real px = o1[0] - o2[0], py = o1[1] - o2[1], pz = o1[2] - o2[2];
        load9(&F.T1toVxfMin[jr], m1); load9(&F.VytoVxfMin[jr], m2);
        mv3(m1, dtT1, o1); mv3(m2, dyV1, o2);
        DxVx[3] = o1[0] - o2[0]; DxVy[3] = o1[1] - o2[1]; DxVz[3] = o1[2] - o2[2];
        DxVx[4] = px; DxVy[4] = py; DxVz[4] = pz;
      }
      real dxV1[3] = { DxVx[3], DxVy[3], DxVz[3] }, dxV2[3] = { DxVx[4], DxVy[4], DxVz[4] };
      load9(&F.Vx2Vz2[jr], m1); load9(&F.Vy2Vz2[jr], m2);
      mv3(m1, dxV2, o1); mv3(m2, dyV2, o2);
      DzVx[4] = o1[0] + o2[0]; DzVy[4] = o1[1] + o2[1]; DzVz[4] = o1[2] + o2[2];
      load9(&F.Vx2Vz1[jr], m1); load9(&F.Vy2Vz1[jr], m2);
      mv3(m1, dxV1, o1); mv3(m2, dyV1, o2);
      DzVx[3] = o1[0] + o2[0]; DzVy[3] = o1[1] + o2[1]; DzVz[3] = o1[2] + o2[2];
    }
    if (S->isfree == 1 && (km == 1 || km == 2)) {
      for (int m = 0; m < 2; m++) {
        const real *ax = fVx + pf + m*ns, *ay = fVy + pf + m*ns, *az = fVz + pf + m*ns;
        int q = 3 + m;
        if (km == 1) { DzVx[q] = mac22(ax,ny,kdir); DzVy[q] = mac22(ay,ny,kdir); DzVz[q] = mac22(az,ny,kdir); }
        else { DzVx[q] = mac24(ax,ny,kdir); DzVy[q] = mac24(ay,ny,kdir); DzVz[q] = mac24(az,ny,kdir); }
      }
      if (S->imethod == 1) {
        real dxV[3], dyV1[3] = { DyVx[3], DyVy[3], DyVz[3] }, dzV1[3] = { DzVx[3], DzVy[3], DzVz[3] };
        real dyV2[3] = { DyVx[4], DyVy[4], DyVz[4] }, dzV2[3] = { DzVx[4], DzVy[4], DzVz[4] };
        if (idir == 1) {
          dxV[0] = DxVx[4]; dxV[1] = DxVy[4]; dxV[2] = DxVz[4];
          load9(&F.P2M1[ix9], m1); load9(&F.P2M2[ix9], m2); load9(&F.P2M3[ix9], m3);
          load9(&F.P2M4[ix9], m4); load9(&F.P2M5[ix9], m5);
          mv3(m1, dxV, o1); mv3(m2, dyV2, o2); mv3(m3, dzV2, o3); mv3(m4, dyV1, o4); mv3(m5, dzV1, o5);
          DxVx[3] = o1[0] + o2[0] + o3[0] - o4[0] - o5[0];
          DxVy[3] = o1[1] + o2[1] + o3[1] - o4[1] - o5[1];
          DxVz[3] = o1[2] + o2[2] + o3[2] - o4[2] - o5[2];
        } else {
          dxV[0] = DxVx[3]; dxV[1] = DxVy[3]; dxV[2] = DxVz[3];
          load9(&F.M2P1[ix9], m1); load9(&F.M2P2[ix9], m2); load9(&F.M2P3[ix9], m3);
          load9(&F.M2P4[ix9], m4); load9(&F.M2P5[ix9], m5);
          mv3(m1, dxV, o1); mv3(m2, dyV1, o2); mv3(m3, dzV1, o3); mv3(m4, dyV2, o4); mv3(m5, dzV2, o5);
          DxVx[4] = o1[0] + o2[0] + o3[0] - o4[0] - o5[0];
          DxVy[4] = o1[1] + o2[1] + o3[1] - o4[1] - o5[1];
          DxVz[4] = o1[2] + o2[2] + o3[2] - o4[2] - o5[2];
        }
      }
      if (S->imethod == 2) {
        get_dtT1();
        real dy[3], dzz[3];
        dy[0] = DyVx[4]; dy[1] = DyVy[4]; dy[2] = DyVz[4]; dzz[0] = DzVx[4]; dzz[1] = DzVy[4]; dzz[2] = DzVz[4];
        load9(&F.T1toVxPlus[ix9], m1); load9(&F.VytoVxPlus[ix9], m2); load9(&F.VztoVxPlus[ix9], m3);
        mv3(m1, dtT1, o1); mv3(m2, dy, o2); mv3(m3, dzz, o3);
        real px = o1[0] - o2[0] - o3[0], py = o1[1] - o2[1] - o3[1], pz = o1[2] - o2[2] - o3[2];
        dy[0] = DyVx[3]; dy[1] = DyVy[3]; dy[2] = DyVz[3]; dzz[0] = DzVx[3]; dzz[1] = DzVy[3]; dzz[2] = DzVz[3];
        load9(&F.T1toVxMin[ix9], m1); load9(&F.VytoVxMin[ix9], m2); load9(&F.VztoVxMin[ix9], m3);
        mv3(m1, dtT1, o1); mv3(m2, dy, o2); mv3(m3, dzz, o3);
        DxVx[3] = o1[0] - o2[0] - o3[0]; DxVy[3] = o1[1] - o2[1] - o3[1]; DxVz[3] = o1[2] - o2[2] - o3[2];
        DxVx[4] = px; DxVy[4] = py; DxVz[4] = pz;
      }
    }
    // fault traction rates f_hT2, f_hT3 on both sides
    for (int side = 0; side < 2; side++) {
      int q = 3 + side;
      real v1[3] = { DxVx[q], DxVy[q], DxVz[q] }, v2[3] = { DyVx[q], DyVy[q], DyVz[q] }, v3[3] = { DzVx[q], DzVy[q], DzVz[q] };
      real g1[3], g2[3], g3[3];
      const std::vector<real> *A2[3] = { side ? &F.D21_2 : &F.D21_1, side ? &F.D22_2 : &F.D22_1, side ? &F.D23_2 : &F.D23_1 };
      const std::vector<real> *A3[3] = { side ? &F.D31_2 : &F.D31_1, side ? &F.D32_2 : &F.D32_1, side ? &F.D33_2 : &F.D33_1 };
      real *fh = frhs + side*ns;
      load9(&(*A2[0])[ix9], m1); load9(&(*A2[1])[ix9], m2); load9(&(*A2[2])[ix9], m3);
      mv3(m1, v1, g1); mv3(m2, v2, g2); mv3(m3, v3, g3);
      fh[FT2X*2*ns+pf] = g1[0] + g2[0] + g3[0];
      fh[FT2Y*2*ns+pf] = g1[1] + g2[1] + g3[1];
      fh[FT2Z*2*ns+pf] = g1[2] + g2[2] + g3[2];
      load9(&(*A3[0])[ix9], m1); load9(&(*A3[1])[ix9], m2); load9(&(*A3[2])[ix9], m3);
      mv3(m1, v1, g1); mv3(m2, v2, g2); mv3(m3, v3, g3);
      fh[FT3X*2*ns+pf] = g1[0] + g2[0] + g3[0];
      fh[FT3Y*2*ns+pf] = g1[1] + g2[1] + g3[1];
      fh[FT3Z*2*ns+pf] = g1[2] + g2[2] + g3[2];
    }
    // points across the fault from the split node: E,F,G (F variant) or C,B,A (B variant)
    if (idir == 1) {
      size_t a = P(i0-1), b = P(i0-2), c3 = P(i0-3), d4 = P(i0-4);
      const real *VV[3] = { Vx, Vy, Vz }, *FF[3] = { fVx, fVy, fVz };
      real *DX[3] = { DxVx, DxVy, DxVz };
      for (int c = 0; c < 3; c++) {
        DX[c][2] = (FF[c][pf] - VV[c][a]);
        real v3[3] = { VV[c][b], VV[c][a], FF[c][pf] };
        DX[c][1] = vec24(v3, 1);
        real v5[5] = { VV[c][d4], VV[c][c3], VV[c][b], VV[c][a], FF[c][pf] };
        DX[c][0] = vec_drp(v5, 1);
      }
    } else {
      size_t a = P(i0+1), b = P(i0+2), c3 = P(i0+3), d4 = P(i0+4);
      const real *VV[3] = { Vx, Vy, Vz }, *FF[3] = { fVx, fVy, fVz };
      real *DX[3] = { DxVx, DxVy, DxVz };
      for (int c = 0; c < 3; c++) {
        DX[c][5] = (VV[c][a] - FF[c][pf+ns]);
        real v3[3] = { FF[c][pf+ns], VV[c][a], VV[c][b] };
        DX[c][6] = vec24(v3, 0);
        real v5[5] = { FF[c][pf+ns], VV[c][a], VV[c][b], VV[c][c3], VV[c][d4] };
        DX[c][7] = vec_drp(v5, 0);
      }
    }
    // stress RHS at i0-3..i0+3 (not i0)
    for (int n = 0; n < 8; n++) {
      int m = n < 4 ? n - 3 : n - 4;
      if (m == 0) continue;
      size_t p = P(i0+m);
      const real *ax = Vx + p, *ay = Vy + p, *az = Vz + p;
      DyVx[n] = macdrp(ax,sy,jdir); DyVy[n] = macdrp(ay,sy,jdir); DyVz[n] = macdrp(az,sy,jdir);
      DzVx[n] = macdrp(ax,sz,kdir); DzVy[n] = macdrp(ay,sz,kdir); DzVz[n] = macdrp(az,sz,kdir);
      size_t idx = ((size_t)(i0+m) + (size_t)jj*S->siz_iy)*9;
      if (S->isfree == 1 && km == 0) {
        const real *X = &S->matVx2Vz[idx], *Y = &S->matVy2Vz[idx];
        DzVx[n] = X[0]*DxVx[n] + X[1]*DxVy[n] + X[2]*DxVz[n] + Y[0]*DyVx[n] + Y[1]*DyVy[n] + Y[2]*DyVz[n];
        DzVy[n] = X[3]*DxVx[n] + X[4]*DxVy[n] + X[5]*DxVz[n] + Y[3]*DyVx[n] + Y[4]*DyVy[n] + Y[5]*DyVz[n];
        DzVz[n] = X[6]*DxVx[n] + X[7]*DxVy[n] + X[8]*DxVz[n] + Y[6]*DyVx[n] + Y[7]*DyVy[n] + Y[8]*DyVz[n];
      }
      if (S->isfree == 1 && km == 1) { DzVx[n] = mac22(ax,sz,kdir); DzVy[n] = mac22(ay,sz,kdir); DzVz[n] = mac22(az,sz,kdir); }
      if (S->isfree == 1 && km == 2) { DzVx[n] = mac24(ax,sz,kdir); DzVy[n] = mac24(ay,sz,kdir); DzVz[n] = mac24(az,sz,kdir); }
      real lam = S->lam[p], mu = S->mu[p];
      real lam2mu = lam + 2.0*mu;
      real xix = S->M(1)[p], xiy = S->M(2)[p], xiz = S->M(3)[p];
      real etx = S->M(4)[p], ety = S->M(5)[p], etz = S->M(6)[p];
      real ztx = S->M(7)[p], zty = S->M(8)[p], ztz = S->M(9)[p];
      h[TXX*ic+p] = lam2mu*(xix*DxVx[n] + etx*DyVx[n] + ztx*DzVx[n])
                  + lam*(xiy*DxVy[n] + ety*DyVy[n] + zty*DzVy[n] + xiz*DxVz[n] + etz*DyVz[n] + ztz*DzVz[n]);
      h[TYY*ic+p] = lam2mu*(xiy*DxVy[n] + ety*DyVy[n] + zty*DzVy[n])
                  + lam*(xix*DxVx[n] + etx*DyVx[n] + ztx*DzVx[n] + xiz*DxVz[n] + etz*DyVz[n] + ztz*DzVz[n]);
      h[TZZ*ic+p] = lam2mu*(xiz*DxVz[n] + etz*DyVz[n] + ztz*DzVz[n])
                  + lam*(xix*DxVx[n] + etx*DyVx[n] + ztx*DzVx[n] + xiy*DxVy[n] + ety*DyVy[n] + zty*DzVy[n]);
      h[TXY*ic+p] = mu*(xiy*DxVx[n] + xix*DxVy[n] + ety*DyVx[n] + etx*DyVy[n] + zty*DzVx[n] + ztx*DzVy[n]);
      h[TXZ*ic+p] = mu*(xiz*DxVx[n] + xix*DxVz[n] + etz*DyVx[n] + etx*DyVz[n] + ztz*DzVx[n] + ztx*DzVz[n]);
      h[TYZ*ic+p] = mu*(xiz*DxVy[n] + xiy*DxVz[n] + etz*DyVy[n] + ety*DyVz[n] + ztz*DzVy[n] + zty*DzVz[n]);
    }
  }
}

/* RK update helpers: wav_update / wav_update_end (wav_t.cu:219-234),
 * fault_wav_update{,_end} (fault_wav_t.cu:319-366) */
void axpy_to(size_t n, real coef, real *out, const real *a, const real *b) {
#pragma omp parallel for
  for (size_t q = 0; q < n; q++) out[q] = a[q] + coef*b[q];
}
void axpy_acc(size_t n, real coef, real *out, const real *b) {
#pragma omp parallel for
  for (size_t q = 0; q < n; q++) out[q] += coef*b[q];
}
void fault_axpy(oracle_solver *S, Fault &F, real coef, real *out, const real *a, const real *b) {
  const size_t ns = S->siz_slice;
  for (int c = 0; c < 18; c++)
    for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) {
      size_t pf = (size_t)(j+S->nj1) + (size_t)(k+S->nk1)*S->ny;
      if (F.united[pf] != 0) continue;
      size_t q = pf + (size_t)c*ns;
      if (a) out[q] = a[q] + coef*b[q]; else out[q] += coef*b[q];
    }
}

// fault_var_stage_update_gpu (fault_wav_t.cu:291-316)
void fault_stage_out(oracle_solver *S, Fault &F, real coef, int istage) {
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) {
    size_t pf = (size_t)(j+S->nj1) + (size_t)(k+S->nk1)*S->ny;
    if (F.united[pf] != 0) continue;
    real *Tn = F.o(CGFD_FAULT_TN), *Ts1 = F.o(CGFD_FAULT_TS1), *Ts2 = F.o(CGFD_FAULT_TS2);
    if (istage == 0) { Tn[pf] = coef*F.tTn[pf]; Ts1[pf] = coef*F.tTs1[pf]; Ts2[pf] = coef*F.tTs2[pf]; }
    else { Tn[pf] += coef*F.tTn[pf]; Ts1[pf] += coef*F.tTs1[pf]; Ts2[pf] += coef*F.tTs2[pf]; }
  }
}

// fault_var_update_gpu (fault_wav_t.cu:198-264)
void fault_step_out(oracle_solver *S, Fault &F, const real *fend, int it) {
  const size_t ns = S->siz_slice;
  const real dt = S->dt;
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) {
    size_t pf = (size_t)(j+S->nj1) + (size_t)(k+S->nk1)*S->ny;
    if (F.united[pf] != 0) continue;
    real dVx = fend[FVX*2*ns+pf+ns] - fend[FVX*2*ns+pf];
    real dVy = fend[FVY*2*ns+pf+ns] - fend[FVY*2*ns+pf];
    real dVz = fend[FVZ*2*ns+pf+ns] - fend[FVZ*2*ns+pf];
    const real *s1 = &F.vec_s1[pf*3], *s2 = &F.vec_s2[pf*3];
    real Vs1 = dVx*s1[0] + dVy*s1[1] + dVz*s1[2];
    real Vs2 = dVx*s2[0] + dVy*s2[1] + dVz*s2[2];
    real Vs = std::sqrt(Vs2*Vs2 + Vs1*Vs1);
    F.o(CGFD_FAULT_VS)[pf] = Vs; F.o(CGFD_FAULT_VS1)[pf] = Vs1; F.o(CGFD_FAULT_VS2)[pf] = Vs2;
    F.o(CGFD_FAULT_SLIP)[pf] += Vs*dt; F.o(CGFD_FAULT_SLIP1)[pf] += Vs1*dt; F.o(CGFD_FAULT_SLIP2)[pf] += Vs2*dt;
    F.hT1x[pf] = (F.T1x[pf+3*ns] - F.mT1x[pf])/dt;
    F.hT1y[pf] = (F.T1y[pf+3*ns] - F.mT1y[pf])/dt;
    F.hT1z[pf] = (F.T1z[pf+3*ns] - F.mT1z[pf])/dt;
    F.mT1x[pf] = F.T1x[pf+3*ns]; F.mT1y[pf] = F.T1y[pf+3*ns]; F.mT1z[pf] = F.T1z[pf+3*ns];
    if (Vs > F.o(CGFD_FAULT_PEAK_VS)[pf]) F.o(CGFD_FAULT_PEAK_VS)[pf] = Vs;
    if (F.t0_flag[pf] == 0 && Vs > 1e-3) {
      F.o(CGFD_FAULT_INIT_T0)[pf] = (it+1)*dt;
      F.t0_flag[pf] = 1;
      F.flag_rup[pf] = 1;
    }
  }
}

// io_recv_keep (io_funcs.cu:428-469) and io_fault_recv_keep (:2313-2351)
void record(oracle_solver *S) {
  if (S->nrec >= S->max_rec) return;
  const size_t ic = S->siz_icmp;
  const real *w = S->W(LPRE);
  for (size_t n = 0; n < S->sta.size(); n++) {
    const Station &R = S->sta[n];
    real Lx2 = R.di, Lx1 = 1.0 - Lx2, Ly2 = R.dj, Ly1 = 1.0 - Ly2, Lz2 = R.dk, Lz1 = 1.0 - Lz2;
    for (int c = 0; c < 9; c++) {
      real b[8];
      for (int q = 0; q < 8; q++) b[q] = w[c*ic + R.idx[q]];
      S->seis[(n*9 + c)*S->max_rec + S->nrec] =
          b[0]*Lx1*Ly1*Lz1 + b[1]*Lx2*Ly1*Lz1 + b[2]*Lx1*Ly2*Lz1 + b[3]*Lx2*Ly2*Lz1
        + b[5]*Lx1*Ly1*Lz2 + b[5]*Lx2*Ly1*Lz2 + b[6]*Lx1*Ly2*Lz2 + b[7]*Lx2*Ly2*Lz2;
    }
  }
  for (size_t n = 0; n < S->fsta.size(); n++) {
    const FStation &R = S->fsta[n];
    Fault &F = S->faults[R.f];
    real Ly2 = R.dj, Ly1 = 1.0 - Ly2, Lz2 = R.dk, Lz1 = 1.0 - Lz2;
    for (int c = 0; c < 9; c++) {
      const real *o = F.o(c);
      S->fseis[(n*9 + c)*S->max_rec + S->nrec] =
          o[R.idx[0]]*Ly1*Lz1 + o[R.idx[1]]*Ly2*Lz1 + o[R.idx[2]]*Ly1*Lz2 + o[R.idx[3]]*Ly2*Lz2;
    }
  }
  S->nrec++;
}

/* -------- exponential sponge: bdry_ablexp_set (bdry_t.cu:453-700),
 *          bdry_cal_abl_len_dh (:329-444), bdry_ablexp_cal_mask (:704-722),
 *          bdry_ablexp_apply_gpu (:764-818) ------------------------------ */
real abl_mask(int i, real vel, real dt, int num_lay, real dh) {
  real len = num_lay * dh;
  int num_step = (int)(len / vel / dt);
  real total_damp = 0;
  for (int n = 0; n < num_step; n++) total_damp += std::pow((n*dt*vel)/len, (real)2.0);
  real alpha = (real)(0.6 / (double)total_damp);
  return std::exp(-alpha * std::pow((real)i/num_lay, (real)2.0));
}

// mean spacing of the block along idim, the reference's loop order
real abl_dh(oracle_solver *S, int i1, int i2, int j1, int j2, int k1, int k2, int idim) {
  double L = 0.0; int num = 0;
  auto seg = [&](size_t a, size_t b) {
    double x0 = S->x3d[a], y0 = S->y3d[a], z0 = S->z3d[a];
    double x1 = S->x3d[b], y1 = S->y3d[b], z1 = S->z3d[b];
    L += std::sqrt((x1-x0)*(x1-x0) + (y1-y0)*(y1-y0) + (z1-z0)*(z1-z0)); num += 1;
  };
  if (idim == 0) {
    for (int k = k1; k <= k2; k++) for (int j = j1; j <= j2; j++) for (int i = i1+1; i <= i2; i++) seg(S->I(i-1,j,k), S->I(i,j,k));
  } else if (idim == 1) {
    for (int k = k1; k <= k2; k++) for (int i = i1; i <= i2; i++) for (int j = j1+1; j <= j2; j++) seg(S->I(i,j-1,k), S->I(i,j,k));
  } else {
    for (int j = j1; j <= j2; j++) for (int i = i1; i <= i2; i++) for (int k = k1+1; k <= k2; k++) seg(S->I(i,j,k-1), S->I(i,j,k));
  }
  return (real)(float)(L / num);
}

void abl_set(oracle_solver *S, const cgfd_config *c) {
  S->abl_Ex.assign(S->nx, 1); S->abl_Ey.assign(S->ny, 1); S->abl_Ez.assign(S->nz, 1);
  const int (&nl)[3][2] = c->ablexp_layers;
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) if (nl[d][s] > 0) S->abl_on = 1;
  const int ni_x = nl[0][0] + nl[0][1], nj_y = nl[1][0] + nl[1][1];
  auto &D = S->abl_blk;
  // x1, x2, y1, y2, z1, z2
  D[0] = { 0, S->ni1, nl[0][0], S->nj1, S->nj, S->nk1, S->nk };
  D[1] = { 0, S->ni2 - nl[0][1] + 1, nl[0][1], S->nj1, S->nj, S->nk1, S->nk };
  D[2] = { 0, S->ni1 + nl[0][0], S->ni - ni_x, S->nj1, nl[1][0], S->nk1, S->nk };
  D[3] = { 0, S->ni1 + nl[0][0], S->ni - ni_x, S->nj2 - nl[1][1] + 1, nl[1][1], S->nk1, S->nk };
  D[4] = { 0, S->ni1 + nl[0][0], S->ni - ni_x, S->nj1 + nl[1][0], S->nj - nj_y, S->nk1, nl[2][0] };
  D[5] = { 0, S->ni1 + nl[0][0], S->ni - ni_x, S->nj1 + nl[1][0], S->nj - nj_y, S->nk2 - nl[2][1] + 1, nl[2][1] };
  for (int n = 0; n < 6; n++) {
    auto &B = D[n];
    if (!(B.ni > 0 && B.nj > 0 && B.nk > 0)) continue;
    B.enable = 1;
    const int d = n / 2, s = n % 2;
    real dh = abl_dh(S, B.ni1, B.ni1 + B.ni - 1, B.nj1, B.nj1 + B.nj - 1, B.nk1, B.nk1 + B.nk - 1, d);
    real vel = c->ablexp_ref_vel[d][s];
    const int lo = d == 0 ? B.ni1 : (d == 1 ? B.nj1 : B.nk1), cnt = d == 0 ? B.ni : (d == 1 ? B.nj : B.nk);
    std::vector<real> &E = d == 0 ? S->abl_Ex : (d == 1 ? S->abl_Ey : S->abl_Ez);
    for (int m = lo; m < lo + cnt; m++)
      E[m] = abl_mask(s == 0 ? cnt - (m - lo) : m - lo + 1, vel, S->dt, cnt, dh);
  }
}

void abl_apply(oracle_solver *S, real *w) {
  const size_t ic = S->siz_icmp;
  for (int n = 0; n < 6; n++) {
    const auto &B = S->abl_blk[n];
    if (!B.enable) continue;
    for (int iz = 0; iz < B.nk; iz++) for (int iy = 0; iy < B.nj; iy++) for (int ix = 0; ix < B.ni; ix++) {
      size_t p = S->I(ix + B.ni1, iy + B.nj1, iz + B.nk1);
      real mask = (S->abl_Ex[ix+B.ni1] < S->abl_Ey[iy+B.nj1]) ? S->abl_Ex[ix+B.ni1] : S->abl_Ey[iy+B.nj1];
      if (mask > S->abl_Ez[iz+B.nk1]) mask = S->abl_Ez[iz+B.nk1];
      for (int c = 0; c < 9; c++) w[p + c*ic] *= mask;
    }
  }
}

/* -------- surface peak motion: PG_calcu_gpu (wav_t.cu:138-216) ---------- */
void pg_calc(oracle_solver *S, const real *w_end, const real *w_pre) {
  const size_t ic = S->siz_icmp, n = S->siz_iz;
  const real dt = S->dt;
  real *PG = S->pg.data(), *Dx = S->dis.data(), *Dy = Dx + n, *Dz = Dx + 2*n;
  for (int iy = 0; iy < S->nj; iy++) for (int ix = 0; ix < S->ni; ix++) {
    const size_t p = S->I(ix + S->ni1, iy + S->nj1, S->nk2), q = (size_t)(ix + S->ni1) + (size_t)(iy + S->nj1)*S->siz_iy;
    const real vx1 = w_end[VX*ic+p], vy1 = w_end[VY*ic+p], vz1 = w_end[VZ*ic+p];
    const real vx0 = w_pre[VX*ic+p], vy0 = w_pre[VY*ic+p], vz0 = w_pre[VZ*ic+p];
    real Ax = std::fabs((vx1-vx0)/dt), Ay = std::fabs((vy1-vy0)/dt), Az = std::fabs((vz1-vz0)/dt);
    // the reference's 0.5 is a double constant
    Dx[q] = (real)((double)Dx[q] + 0.5*(double)(vx1+vx0)*(double)dt);
    Dy[q] = (real)((double)Dy[q] + 0.5*(double)(vy1+vy0)*(double)dt);
    Dz[q] = (real)((double)Dz[q] + 0.5*(double)(vz1+vz0)*(double)dt);
    const real val[15] = {
      std::sqrt(vx1*vx1 + vy1*vy1 + vz1*vz1), std::sqrt(vx1*vx1 + vy1*vy1),
      std::fabs(vx1), std::fabs(vy1), std::fabs(vz1),
      std::sqrt(Ax*Ax + Ay*Ay + Az*Az), std::sqrt(Ax*Ax + Ay*Ay), Ax, Ay, Az,
      std::sqrt(Dx[q]*Dx[q] + Dy[q]*Dy[q] + Dz[q]*Dz[q]), std::sqrt(Dx[q]*Dx[q] + Dy[q]*Dy[q]),
      std::fabs(Dx[q]), std::fabs(Dy[q]), std::fabs(Dz[q]) };
    for (int c = 0; c < 15; c++) if (PG[c*n + q] < val[c]) PG[c*n + q] = val[c];
  }
}

/* one time step: drv_rk_curv_col.cu:209-636 */
void step(oracle_solver *S) {
  const int it = S->it;
  record(S);
  const int ipair = it % 8;
  const size_t nlev = 9*S->siz_icmp;
  const real dt = S->dt;
  for (int istage = 0; istage < 4; istage++) {
    const int idir = (FD_FLAGS[ipair][0] + istage) % 2;
    const int jdir = (FD_FLAGS[ipair][1] + istage) % 2;
    const int kdir = (FD_FLAGS[ipair][2] + istage) % 2;
    const int curl = istage == 0 ? LPRE : LTMP;
    real *w_cur = S->W(curl), *w_rhs = S->W(LRHS), *w_pre = S->W(LPRE), *w_tmp = S->W(LTMP), *w_end = S->W(LEND);
    // PML "cur" pointer (drv_rk_curv_col.cu:241-266)
    for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) S->pml[d][s].cur = S->pml[d][s].lvl[curl];
    for (auto &F : S->faults) {
      real *f_cur = F.lev(curl), *f_rhs = F.lev(LRHS), *f_pre = F.lev(LPRE);
      wave2fault(S, F, w_cur, w_rhs, f_cur, f_rhs);
      trial(S, F, w_cur, f_cur, f_pre, jdir, kdir);
      fault2wave(S, F, w_cur, f_cur);
    }
    rhs_inner(S, w_cur, w_rhs, idir, jdir, kdir);
    if (S->isfree) {
      rhs_timg(S, w_cur, w_rhs, idir, jdir, kdir);
      rhs_vlow(S, w_cur, w_rhs, idir, jdir, kdir);
    }
    if (S->pml_on) rhs_pml(S, w_cur, w_rhs, idir, jdir, kdir);
    for (auto &F : S->faults) {
      real *f_cur = F.lev(curl), *f_rhs = F.lev(LRHS);
      rhs_fault_velo(S, F, w_cur, w_rhs, f_cur, f_rhs, idir, jdir, kdir);
      rhs_fault_stress(S, F, w_cur, w_rhs, f_cur, f_rhs, idir, jdir, kdir);
    }
    // RK
    if (istage == 0) {
      real ca = RK_A[istage]*dt, cb = RK_B[istage]*dt;
      axpy_to(nlev, ca, w_tmp, w_pre, w_rhs);
      for (auto &F : S->faults) {
        fault_axpy(S, F, ca, F.lev(LTMP), F.lev(LPRE), F.lev(LRHS));
        fault2wave(S, F, w_tmp, F.lev(LTMP));
      }
      for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
        PmlFace &P = S->pml[d][s]; if (!P.on) continue;
        axpy_to(9*P.siz, ca, P.lev(LTMP), P.lev(LPRE), P.lev(LRHS));
      }
      axpy_to(nlev, cb, w_end, w_pre, w_rhs);
      for (auto &F : S->faults) fault_axpy(S, F, cb, F.lev(LEND), F.lev(LPRE), F.lev(LRHS));
      for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
        PmlFace &P = S->pml[d][s]; if (!P.on) continue;
        axpy_to(9*P.siz, cb, P.lev(LEND), P.lev(LPRE), P.lev(LRHS));
      }
    } else if (istage < 3) {
      real ca = RK_A[istage]*dt, cb = RK_B[istage]*dt;
      axpy_to(nlev, ca, w_tmp, w_pre, w_rhs);
      for (auto &F : S->faults) {
        fault_axpy(S, F, ca, F.lev(LTMP), F.lev(LPRE), F.lev(LRHS));
        fault2wave(S, F, w_tmp, F.lev(LTMP));
      }
      for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
        PmlFace &P = S->pml[d][s]; if (!P.on) continue;
        axpy_to(9*P.siz, ca, P.lev(LTMP), P.lev(LPRE), P.lev(LRHS));
      }
      axpy_acc(nlev, cb, w_end, w_rhs);
      for (auto &F : S->faults) fault_axpy(S, F, cb, F.lev(LEND), nullptr, F.lev(LRHS));
      for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
        PmlFace &P = S->pml[d][s]; if (!P.on) continue;
        axpy_acc(9*P.siz, cb, P.lev(LEND), P.lev(LRHS));
      }
    } else {
      real cb = RK_B[istage]*dt;
      axpy_acc(nlev, cb, w_end, w_rhs);
      for (auto &F : S->faults) {
        fault_axpy(S, F, cb, F.lev(LEND), nullptr, F.lev(LRHS));
        fault2wave(S, F, w_end, F.lev(LEND));
      }
      for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
        PmlFace &P = S->pml[d][s]; if (!P.on) continue;
        axpy_acc(9*P.siz, cb, P.lev(LEND), P.lev(LRHS));
      }
    }
    for (auto &F : S->faults) fault_stage_out(S, F, RK_B[istage], istage);
  }
  // end of step: sponge, surface peaks, fault outputs (drv_rk_curv_col.cu:596-616)
  if (S->abl_on) abl_apply(S, S->W(LEND));
  if (S->isfree) pg_calc(S, S->W(LEND), S->W(LPRE));
  for (auto &F : S->faults) fault_step_out(S, F, F.lev(LEND), it);
  std::swap(S->wl[LPRE], S->wl[LEND]);
  for (auto &F : S->faults) std::swap(F.lvl[LPRE], F.lvl[LEND]);
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) std::swap(S->pml[d][s].lvl[LPRE], S->pml[d][s].lvl[LEND]);
  S->it++;
}

} // namespace

/* ============================== C API =================================== */
extern "C" {

int oracle_real_bytes(void) { return (int)sizeof(real); }

int oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n; return 1;
#endif
}

const char *oracle_last_error(void) { return g_err.c_str(); }

int oracle_create(const cgfd_config *c, oracle_solver **out) {
  if (!c || !out) return set_err(CGFD_ERR_ARG, "null argument");
  *out = nullptr;
  if (c->ni < 8 || c->nj < 8 || c->nk < 8) return set_err(CGFD_ERR_ARG, "grid too small");
  if (c->num_faults < 0 || c->num_faults > CGFD_MAX_FAULTS) return set_err(CGFD_ERR_ARG, "num_faults out of range");
  if (!c->lambda || !c->mu || !c->rho) return set_err(CGFD_ERR_ARG, "medium arrays missing");
  if (c->grid_mode == CGFD_GRID_FAULT_PLANE && (c->num_faults < 1 || !c->fault_x || !c->fault_y || !c->fault_z))
    return set_err(CGFD_ERR_ARG, "fault-plane grid needs fault surfaces");
  if (c->grid_mode == CGFD_GRID_IMPORT && (!c->x3d || !c->y3d || !c->z3d))
    return set_err(CGFD_ERR_ARG, "grid import needs coordinates");
  oracle_solver *S = new oracle_solver();
  S->ni = c->ni; S->nj = c->nj; S->nk = c->nk;
  S->nx = S->ni + 6; S->ny = S->nj + 6; S->nz = S->nk + 6;
  S->ni1 = 3; S->ni2 = 3 + S->ni - 1; S->nj1 = 3; S->nj2 = 3 + S->nj - 1; S->nk1 = 3; S->nk2 = 3 + S->nk - 1;
  S->siz_iy = S->nx; S->siz_iz = (size_t)S->nx*S->ny; S->siz_icmp = S->siz_iz*S->nz;
  S->siz_slice = (size_t)S->ny*S->nz;
  S->dt = c->dt; S->imethod = c->dynamic_method; S->isfree = c->free_surface ? 1 : 0;
  gen_grid(S, c);
  calc_metric(S);
  S->lam.assign(S->siz_icmp, 0); S->mu.assign(S->siz_icmp, 0); S->rho.assign(S->siz_icmp, 0);
  for (int k = 0; k < S->nz; k++) for (int j = 0; j < S->ny; j++) for (int i = 0; i < S->nx; i++) {
    int ci = std::min(std::max(i-3, 0), S->ni-1), cj = std::min(std::max(j-3, 0), S->nj-1), ck = std::min(std::max(k-3, 0), S->nk-1);
    size_t src = (size_t)ci + (size_t)S->ni*((size_t)cj + (size_t)S->nj*ck);
    size_t p = S->I(i,j,k);
    S->lam[p] = c->lambda[src]; S->mu[p] = c->mu[src]; S->rho[p] = c->rho[src];
  }
  calc_dtmax(S);
  if (c->check_stability && S->dt > S->dtmax) {
    char b[160]; snprintf(b, sizeof b, "dt=%g above the CFL limit %g", (double)S->dt, (double)S->dtmax);
    delete S; return set_err(CGFD_ERR_DT, b);
  }
  int margin = c->welded_margin;
  for (int f = 0; f < c->num_faults; f++) {
    Fault F;
    F.i0 = c->fault_x_index[f] - 1 + 3;
    for (int q = 0; q < 4; q++) F.grid[q] = c->fault_grid[f][q] - 1;
    if (F.i0 < 3 + 4 || F.i0 > S->ni2 - 4) { delete S; return set_err(CGFD_ERR_ARG, "fault_x_index too close to the x sides"); }
    S->faults.push_back(F);
  }
  for (int f = 0; f < c->num_faults; f++) fault_coef(S, S->faults[f]);
  for (int f = 0; f < c->num_faults; f++) fault_set(S, S->faults[f], c, f, margin);
  pml_set(S, c);
  abl_set(S, c);
  if (S->isfree) free_set(S);
  if (S->isfree) { S->pg.assign(15*S->siz_iz, 0); S->dis.assign(3*S->siz_iz, 0); }
  for (size_t q = 0; q < S->siz_icmp; q++) S->rho[q] = S->rho[q] > 1e-10 ? 1.0/S->rho[q] : 0.0;
  for (int l = 0; l < 4; l++) S->w[l].assign(9*S->siz_icmp, 0);
  S->max_rec = c->max_records > 0 ? c->max_records : 0;
  for (int n = 0; n < c->num_stations; n++) {
    Station R;
    float gx = c->station_ijk[3*n], gy = c->station_ijk[3*n+1], gz = c->station_ijk[3*n+2];
    int ix = (int)gx, iy = (int)gy, iz = (int)gz;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= S->ni || iy >= S->nj || iz >= S->nk) continue;
    R.i = ix + 3; R.j = iy + 3; R.k = iz + 3;
    R.di = gx - ix; R.dj = gy - iy; R.dk = gz - iz;
    for (int q = 0; q < 8; q++) R.idx[q] = S->I(R.i + (q & 1), R.j + ((q >> 1) & 1), R.k + ((q >> 2) & 1));
    S->sta.push_back(R);
  }
  for (int n = 0; n < c->num_fault_stations; n++) {
    FStation R;
    R.f = c->fault_station_fault[n];
    float gy = c->fault_station_jk[2*n], gz = c->fault_station_jk[2*n+1];
    int iy = (int)std::floor(gy), iz = (int)std::floor(gz);
    if (R.f < 0 || R.f >= c->num_faults || iy < 0 || iz < 0 || iy >= S->nj || iz >= S->nk) continue;
    R.j = iy + 3; R.k = iz + 3; R.dj = gy - iy; R.dk = gz - iz;
    R.idx[0] = (size_t)R.j + (size_t)R.k*S->ny;     R.idx[1] = (size_t)(R.j+1) + (size_t)R.k*S->ny;
    R.idx[2] = (size_t)R.j + (size_t)(R.k+1)*S->ny; R.idx[3] = (size_t)(R.j+1) + (size_t)(R.k+1)*S->ny;
    S->fsta.push_back(R);
  }
  S->seis.assign(S->sta.size()*9*(size_t)S->max_rec, 0);
  S->fseis.assign(S->fsta.size()*9*(size_t)S->max_rec, 0);
  *out = S;
  return CGFD_OK;
}

int oracle_run(oracle_solver *S, int n) {
  if (!S || n < 0) return set_err(CGFD_ERR_ARG, "bad argument");
  for (int q = 0; q < n; q++) step(S);
  return CGFD_OK;
}

int oracle_get_fault(oracle_solver *S, int f, int field, float *out) {
  if (!S || !out || f < 0 || f >= (int)S->faults.size() || field < 0 || field >= CGFD_FAULT_NFIELD)
    return set_err(CGFD_ERR_ARG, "bad argument");
  Fault &F = S->faults[f];
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++)
    out[(size_t)k*S->nj + j] = (float)F.o(field)[(size_t)(j+3) + (size_t)(k+3)*S->ny];
  return CGFD_OK;
}

int oracle_get_stations(oracle_solver *S, float *out, int *nrec) {
  if (!S) return set_err(CGFD_ERR_ARG, "bad argument");
  if (nrec) *nrec = S->nrec;
  if (out) for (size_t n = 0; n < S->sta.size()*9; n++)
    for (int t = 0; t < S->nrec; t++) out[n*S->nrec + t] = (float)S->seis[n*S->max_rec + t];
  return CGFD_OK;
}

int oracle_get_fault_stations(oracle_solver *S, float *out, int *nrec) {
  if (!S) return set_err(CGFD_ERR_ARG, "bad argument");
  if (nrec) *nrec = S->nrec;
  if (out) for (size_t n = 0; n < S->fsta.size()*9; n++)
    for (int t = 0; t < S->nrec; t++) out[n*S->nrec + t] = (float)S->fseis[n*S->max_rec + t];
  return CGFD_OK;
}

int oracle_get_wavefield(oracle_solver *S, int cmp, float *out) {
  if (!S || !out || cmp < 0 || cmp >= 9) return set_err(CGFD_ERR_ARG, "bad argument");
  const real *w = S->W(LPRE) + cmp*S->siz_icmp;
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) for (int i = 0; i < S->ni; i++)
    out[(size_t)i + (size_t)S->ni*((size_t)j + (size_t)S->nj*k)] = (float)w[S->I(i+3,j+3,k+3)];
  return CGFD_OK;
}

int oracle_set_wavefield(oracle_solver *S, int cmp, const float *in) {
  if (!S || !in || cmp < 0 || cmp >= 9) return set_err(CGFD_ERR_ARG, "bad argument");
  real *w = S->W(LPRE) + cmp*S->siz_icmp;
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) for (int i = 0; i < S->ni; i++)
    w[S->I(i+3,j+3,k+3)] = in[(size_t)i + (size_t)S->ni*((size_t)j + (size_t)S->nj*k)];
  return CGFD_OK;
}

int oracle_get_metric(oracle_solver *S, int cmp, float *out) {
  if (!S || !out || cmp < 0 || cmp >= 10) return set_err(CGFD_ERR_ARG, "bad argument");
  const real *m = S->M(cmp);
  for (int k = 0; k < S->nk; k++) for (int j = 0; j < S->nj; j++) for (int i = 0; i < S->ni; i++)
    out[(size_t)i + (size_t)S->ni*((size_t)j + (size_t)S->nj*k)] = (float)m[S->I(i+3,j+3,k+3)];
  return CGFD_OK;
}

int oracle_get_surface_peaks(oracle_solver *S, float *out) {
  if (!S || !out) return set_err(CGFD_ERR_ARG, "bad argument");
  if (!S->isfree) return set_err(CGFD_ERR_ARG, "no free surface");
  for (int c = 0; c < 15; c++) for (int j = 0; j < S->nj; j++) for (int i = 0; i < S->ni; i++)
    out[((size_t)c*S->nj + j)*S->ni + i] = (float)S->pg[c*S->siz_iz + (size_t)(i+3) + (size_t)(j+3)*S->siz_iy];
  return CGFD_OK;
}

int oracle_dt_max(oracle_solver *S, float *d) { if (!S || !d) return CGFD_ERR_ARG; *d = (float)S->dtmax; return CGFD_OK; }

void oracle_destroy(oracle_solver *S) { delete S; }

} // extern "C"
