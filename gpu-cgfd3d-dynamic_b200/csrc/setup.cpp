// setup.cpp -- host set-up of a forward problem.  See setup.h.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace cgfd {
namespace {

typedef double M3[3][3];

void inv3(const M3 a, M3 r) {
  double c00 = a[1][1]*a[2][2] - a[2][1]*a[1][2];
  double c01 = a[2][1]*a[0][2] - a[0][1]*a[2][2];
  double c02 = a[0][1]*a[1][2] - a[0][2]*a[1][1];
  double c10 = a[1][2]*a[2][0] - a[1][0]*a[2][2];
  double c11 = a[0][0]*a[2][2] - a[2][0]*a[0][2];
  double c12 = a[1][0]*a[0][2] - a[0][0]*a[1][2];
  double c20 = a[1][0]*a[2][1] - a[1][1]*a[2][0];
  double c21 = a[2][0]*a[0][1] - a[0][0]*a[2][1];
  double c22 = a[0][0]*a[1][1] - a[0][1]*a[1][0];
  double id = 1.0 / (c00*a[0][0] + c01*a[1][0] + c02*a[2][0]);
  double t[3][3] = {{c00, c01, c02}, {c10, c11, c12}, {c20, c21, c22}};
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) r[i][j] = t[i][j] * id;
}
void mul3(const M3 a, const M3 b, M3 c) {
  double t[3][3];
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
    t[i][j] = a[i][0]*b[0][j] + a[i][1]*b[1][j] + a[i][2]*b[2][j];
  std::memcpy(c, t, sizeof(t));
}
void cross(const double *a, const double *b, double *c) {
  c[0] = a[1]*b[2] - a[2]*b[1]; c[1] = a[2]*b[0] - a[0]*b[2]; c[2] = a[0]*b[1] - a[1]*b[0];
}
double dot(const double *a, const double *b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
double nrm(const double *a) { return std::sqrt(dot(a, a)); }

// Traction-rate block: the jac-weighted traction on the e_a face produced by
// a velocity gradient along e_b in an isotropic medium,
//   D_ab = jac * ( lam e_a (x) e_b + mu e_b (x) e_a + mu (e_a . e_b) I ),
// the closed form of the 9-term expressions of fault_coef_cal
// (src/forward/fault_info.cu:180-300).
void dblock(const double *ea, const double *eb, double lam, double mu, double jac, M3 d) {
  double ab = dot(ea, eb);
  for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++)
    d[r][c] = jac * (lam*ea[r]*eb[c] + mu*eb[r]*ea[c] + (r == c ? mu*ab : 0.0));
}

void put9(const M3 m, float *dst) { for (int q = 0; q < 9; q++) dst[q] = (float)m[q/3][q%3]; }

// linear extrapolation into the ghost layers, in the reference's order and
// float arithmetic (geometric_symmetry, src/forward/gd_t.cu:666-759)
template <class IDX>
void extrapolate(float *v, int nx, int ny, int nz, IDX I) {
  const int a1 = NG, a2 = nx - NG - 1, b1 = NG, b2 = ny - NG - 1, c1 = NG, c2 = nz - NG - 1;
  for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) {
    for (int i = 0; i < a1; i++) v[I(i,j,k)] = 2*v[I(a1,j,k)] - v[I(2*a1-i,j,k)];
    for (int i = a2+1; i < nx; i++) v[I(i,j,k)] = 2*v[I(a2,j,k)] - v[I(2*a2-i,j,k)];
  }
  for (int k = 0; k < nz; k++) for (int i = 0; i < nx; i++) {
    for (int j = 0; j < b1; j++) v[I(i,j,k)] = 2*v[I(i,b1,k)] - v[I(i,2*b1-j,k)];
    for (int j = b2+1; j < ny; j++) v[I(i,j,k)] = 2*v[I(i,b2,k)] - v[I(i,2*b2-j,k)];
  }
  for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++) {
    for (int k = 0; k < c1; k++) v[I(i,j,k)] = 2*v[I(i,j,c1)] - v[I(i,j,2*c1-k)];
    for (int k = c2+1; k < nz; k++) v[I(i,j,k)] = 2*v[I(i,j,c2)] - v[I(i,j,2*c2-k)];
  }
}

// bdry_ablexp_cal_mask (src/forward/bdry_t.cu:704-722), in its float
// arithmetic: alpha spreads a total damping of 0.6 over the steps a wave
// at `vel` takes to cross the layer
float ablexp_mask(int i, float vel, float dt, int num_lay, float dh) {
  const float len = num_lay * dh;
  const int num_step = (int)(len / vel / dt);
  float total = 0.0f;
  for (int n = 0; n < num_step; n++) total += powf((n * dt * vel) / len, 2.0f);
  const float alpha = (float)(0.6 / total);
  return expf(-alpha * powf((float)i / num_lay, 2.0f));
}

}  // namespace

int build_setup(const cgfd_config *c, HostSetup &S, std::string &msg) {
  if (c->ni < 12 || c->nj < 12 || c->nk < 12) { msg = "grid must have at least 12 points per axis"; return CGFD_ERR_ARG; }
  if (c->num_faults < 0 || c->num_faults > CGFD_MAX_FAULTS) { msg = "num_faults out of range"; return CGFD_ERR_ARG; }
  if (c->dynamic_method != 1 && c->dynamic_method != 2) { msg = "dynamic_method must be 1 or 2"; return CGFD_ERR_ARG; }
  if (!(c->dt > 0.f)) { msg = "dt must be positive"; return CGFD_ERR_ARG; }
  if (!c->lambda || !c->mu || !c->rho) { msg = "medium arrays (lambda, mu, rho) missing"; return CGFD_ERR_ARG; }
  if (c->grid_mode == CGFD_GRID_FAULT_PLANE) {
    if (c->num_faults < 1 || !c->fault_x || !c->fault_y || !c->fault_z) { msg = "fault-plane grid needs fault surfaces"; return CGFD_ERR_ARG; }
  } else if (c->grid_mode == CGFD_GRID_IMPORT) {
    if (!c->x3d || !c->y3d || !c->z3d) { msg = "grid import needs x3d, y3d, z3d"; return CGFD_ERR_ARG; }
  } else { msg = "unknown grid_mode"; return CGFD_ERR_ARG; }
  if (c->num_faults > 0 && (!c->T0x || !c->T0y || !c->T0z || !c->mu_s || !c->mu_d || !c->Dc || !c->C0)) {
    msg = "fault initial stress / friction arrays missing"; return CGFD_ERR_ARG;
  }
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
    int L = c->pml_layers[d][s];
    int n = d == 0 ? c->ni : (d == 1 ? c->nj : c->nk);
    if (L < 0 || L > n / 2 - 1) { msg = "pml_layers out of range"; return CGFD_ERR_ARG; }
    if (L > 0 && !(c->pml_ref_vel[d][s] > 0.f)) { msg = "pml_ref_vel must be positive"; return CGFD_ERR_ARG; }
  }
  {
    bool any_abl = false, any_pml = false;
    for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
      const int L = c->ablexp_layers[d][s];
      const int n = d == 0 ? c->ni : (d == 1 ? c->nj : c->nk);
      if (L < 0 || L > n / 2 - 1) { msg = "ablexp_layers out of range"; return CGFD_ERR_ARG; }
      if (L > 0 && !(c->ablexp_ref_vel[d][s] > 0.f)) { msg = "ablexp_ref_vel must be positive"; return CGFD_ERR_ARG; }
      any_abl |= L > 0;
      any_pml |= c->pml_layers[d][s] > 0;
    }
    if (any_abl && any_pml) { msg = "ablexp and cfspml faces cannot be combined"; return CGFD_ERR_ARG; }
    if (c->free_surface && c->ablexp_layers[2][1] > 0) { msg = "ablexp on the free top face"; return CGFD_ERR_ARG; }
  }

  Grid &g = S.g;
  g.ni = c->ni; g.nj = c->nj; g.nk = c->nk;
  g.nx = g.ni + 2*NG; g.ny = g.nj + 2*NG; g.nz = g.nk + 2*NG;
  {
    // the interior box starts after the left x PML (its layers + 1 points)
    const int ilo = c->pml_layers[0][0] > 0 ? c->pml_layers[0][0] + 1 : 0;
    // 8 points of 16-byte groups per 128-byte line (the double build's
    // 32-byte groups need a multiple of 4, which this also is)
    g.xoff = (8 - (ilo + NG) % 8) % 8;
  }
  g.sy = ((g.nx + g.xoff + 31) / 32) * 32;
  g.sz = g.sy * g.ny;
  g.scmp = g.sz * g.nz;
  S.dt = c->dt; S.imethod = c->dynamic_method; S.isfree = c->free_surface ? 1 : 0;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int ni1 = NG, ni2 = NG + g.ni - 1, nj1 = NG, nj2 = NG + g.nj - 1, nk1 = NG, nk2 = NG + g.nk - 1;
  auto U = [&](int i, int j, int k) { return (size_t)i + (size_t)nx*((size_t)j + (size_t)ny*k); };

  // ---- coordinates (gd_curv_gen_fault, gd_t.cu:402-545) in float --------
  std::vector<float> X((size_t)nx*ny*nz), Y(X.size()), Z(X.size());
  if (c->grid_mode == CGFD_GRID_IMPORT) {
    for (int k = 0; k < g.nk; k++) for (int j = 0; j < g.nj; j++) for (int i = 0; i < g.ni; i++) {
      size_t s = (size_t)i + (size_t)g.ni*((size_t)j + (size_t)g.nj*k), d = U(i+NG, j+NG, k+NG);
      X[d] = c->x3d[s]; Y[d] = c->y3d[s]; Z[d] = c->z3d[s];
    }
  } else {
    const float dh = c->fault_interval;
    const size_t fs = (size_t)g.nj * g.nk;
    auto F = [&](const float *a, int f, int j, int k) { return a[f*fs + (size_t)(j-NG) + (size_t)(k-NG)*g.nj]; };
    const int nf = c->num_faults;
    for (int k = nk1; k <= nk2; k++) for (int j = nj1; j <= nj2; j++) {
      int ia = c->fault_x_index[0] - 1 + NG;
      float x = F(c->fault_x,0,j,k), y = F(c->fault_y,0,j,k), z = F(c->fault_z,0,j,k);
      if (nf == 1) {
        for (int i = ni1; i <= ni2; i++) { size_t p = U(i,j,k); X[p] = x + (i-ia)*dh; Y[p] = y; Z[p] = z; }
        continue;
      }
      for (int i = ni1; i <= ia; i++) { size_t p = U(i,j,k); X[p] = x - (ia-i)*dh; Y[p] = y; Z[p] = z; }
      for (int f = 1; f < nf; f++) {
        int a = c->fault_x_index[f-1] - 1 + NG, b = c->fault_x_index[f] - 1 + NG;
        float xb = F(c->fault_x,f,j,k), yb = F(c->fault_y,f,j,k), zb = F(c->fault_z,f,j,k);
        size_t q = U(a,j,k);
        float dhx = (xb - X[q])/(b-a), dhy = (yb - Y[q])/(b-a), dhz = (zb - Z[q])/(b-a);
        for (int i = a+1; i <= b; i++) { size_t p = U(i,j,k); X[p] = xb - (b-i)*dhx; Y[p] = yb - (b-i)*dhy; Z[p] = zb - (b-i)*dhz; }
      }
      int b = c->fault_x_index[nf-1] - 1 + NG;
      float xb = F(c->fault_x,nf-1,j,k), yb = F(c->fault_y,nf-1,j,k), zb = F(c->fault_z,nf-1,j,k);
      for (int i = b+1; i <= ni2; i++) { size_t p = U(i,j,k); X[p] = xb + (i-b)*dh; Y[p] = yb; Z[p] = zb; }
    }
  }
  extrapolate(X.data(), nx, ny, nz, U);
  extrapolate(Y.data(), nx, ny, nz, U);
  extrapolate(Z.data(), nx, ny, nz, U);
  {
    const size_t np = (size_t)g.ni * g.nj * g.nk;
    S.coords.resize(3 * np);
    for (int k = 0; k < g.nk; k++) for (int j = 0; j < g.nj; j++) for (int i = 0; i < g.ni; i++) {
      const size_t s = (size_t)i + (size_t)g.ni * ((size_t)j + (size_t)g.nj * k), d = U(i+NG, j+NG, k+NG);
      S.coords[s] = X[d]; S.coords[np + s] = Y[d]; S.coords[2 * np + s] = Z[d];
    }
  }

  // ---- metric (gd_curv_metric_cal, gd_t.cu:210-304) ----------------------
  // 6th-order centred differences with the reference's rounded weights
  const double W6[7] = { -0.01666667, 0.15, -0.75, 0.0, 0.75, -0.15, 0.01666667 };
  std::vector<float> Mu((size_t)10 * X.size());   // unpadded metric, then copied
  float *Mp[10];
  for (int q = 0; q < 10; q++) Mp[q] = Mu.data() + (size_t)q * X.size();
  long bad = 0;
#pragma omp parallel for collapse(2) reduction(+:bad)
  for (int k = nk1; k <= nk2; k++) for (int j = nj1; j <= nj2; j++) for (int i = ni1; i <= ni2; i++) {
    size_t p = U(i,j,k);
    long st[3] = { 1, (long)nx, (long)nx*ny };
    double e[3][3];   // e[a] = d(x,y,z)/d(xi_a)
    for (int a = 0; a < 3; a++) {
      double sx = 0, sy = 0, sz = 0;
      for (int m = -3; m <= 3; m++) {
        if (m == 0) continue;
        long o = (long)p + m*st[a];
        sx += W6[m+3]*X[o]; sy += W6[m+3]*Y[o]; sz += W6[m+3]*Z[o];
      }
      e[a][0] = (float)sx; e[a][1] = (float)sy; e[a][2] = (float)sz;
    }
    double g0[3], g1[3], g2[3];
    cross(e[1], e[2], g0); cross(e[2], e[0], g1); cross(e[0], e[1], g2);
    double J = dot(g2, e[2]);
    if (!(J > 0.0)) bad++;
    Mp[MJAC][p] = (float)J;
    for (int q = 0; q < 3; q++) { Mp[MXIX+q][p] = (float)(g0[q]/J); Mp[METX+q][p] = (float)(g1[q]/J); Mp[MZTX+q][p] = (float)(g2[q]/J); }
  }
  if (bad) { msg = "grid has non-positive Jacobian (check axis orientation: z must point up)"; return CGFD_ERR_ARG; }
  for (int q = 0; q < 10; q++) extrapolate(Mp[q], nx, ny, nz, U);

  // ---- medium, ghosts take the nearest interior value --------------------
  std::vector<float> lam(X.size()), mu(X.size()), rho(X.size());
  for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) for (int i = 0; i < nx; i++) {
    int ci = std::min(std::max(i-NG, 0), g.ni-1), cj = std::min(std::max(j-NG, 0), g.nj-1), ck = std::min(std::max(k-NG, 0), g.nk-1);
    size_t s = (size_t)ci + (size_t)g.ni*((size_t)cj + (size_t)g.nj*ck), p = U(i,j,k);
    lam[p] = c->lambda[s]; mu[p] = c->mu[s]; rho[p] = c->rho[s];
    if (!(rho[p] > 0.f) || !(mu[p] >= 0.f) || !(lam[p] + 2.f*mu[p] > 0.f)) { msg = "medium must have rho > 0, mu >= 0, lambda + 2 mu > 0"; return CGFD_ERR_ARG; }
  }

  // ---- stability limit (blk_dt_esti_curv, blk_t.cu:72-151) ---------------
  double dtmax = 1e30;
#pragma omp parallel for collapse(2) reduction(min:dtmax)
  for (int k = nk1; k <= nk2; k++) for (int j = nj1; j <= nj2; j++) for (int i = ni1; i <= ni2; i++) {
    size_t p = U(i,j,k);
    double vp = std::sqrt(((double)lam[p] + 2.0*mu[p]) / rho[p]);
    double p0[3] = { X[p], Y[p], Z[p] }, L = 1e30;
    for (int kk = -1; kk <= 1; kk += 2) for (int jj = -1; jj <= 1; jj += 2) for (int ii = -1; ii <= 1; ii += 2) {
      size_t a = p - ii, b = p - (long)jj*nx, cc = p - (long)kk*nx*ny;
      double p1[3] = { X[a], Y[a], Z[a] }, p2[3] = { X[b], Y[b], Z[b] }, p3[3] = { X[cc], Y[cc], Z[cc] };
      double u[3] = { p2[0]-p1[0], p2[1]-p1[1], p2[2]-p1[2] }, v[3] = { p3[0]-p1[0], p3[1]-p1[1], p3[2]-p1[2] };
      double n[3]; cross(u, v, n);
      double d = std::fabs(dot(n, p0) - dot(n, p1)) / nrm(n);
      L = std::min(L, d);
    }
    dtmax = std::min(dtmax, 1.3 / vp * L);
  }
  S.dtmax = (float)dtmax;
  if (c->check_stability && c->dt > S.dtmax) {
    char b[200]; snprintf(b, sizeof b, "dt=%g exceeds the stability limit %g (CFL 1.3)", (double)c->dt, dtmax);
    msg = b; return CGFD_ERR_DT;
  }

  // ---- metric and medium in the padded device layout (coef_row /
  //      coef_jac of common.h): the Jacobian plane, then per direction d
  //      the groups (e_d.x, e_d.y, e_d.z, lambda | mu | 1/rho) ------------
  S.coef.assign((size_t)13 * g.scmp, 0.f);
  {
    const size_t sc = g.scmp;
    float *jac = S.coef.data(), *grp = S.coef.data() + sc;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const size_t p = U(i,j,k), d = (size_t)g.at(i,j,k);
          const float med[3] = { lam[p], mu[p], rho[p] > 1e-10f ? (float)(1.0 / rho[p]) : 0.f };
          jac[d] = Mp[MJAC][p];
          for (int r = 0; r < 3; r++) {
            float *o = grp + 4 * (r * sc + d);
            o[0] = Mp[MXIX + 3 * r][p]; o[1] = Mp[MXIX + 3 * r + 1][p]; o[2] = Mp[MXIX + 3 * r + 2][p];
            o[3] = med[r];
          }
        }
  }

  // ---- CFS-PML (bdry_pml_set, bdry_t.cu:80-251 and 292-440) --------------
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
    PmlHost &P = S.pml[d][s];
    P.L = c->pml_layers[d][s]; P.on = P.L > 0;
    P.i1 = ni1; P.i2 = ni2; P.j1 = nj1; P.j2 = nj2; P.k1 = nk1; P.k2 = nk2;
    int *lo = d == 0 ? &P.i1 : (d == 1 ? &P.j1 : &P.k1), *hi = d == 0 ? &P.i2 : (d == 1 ? &P.j2 : &P.k2);
    if (s == 0) *hi = *lo + P.L; else *lo = *hi - P.L;
    if (!P.on) continue;
    // mean spacing along the normal inside the face region
    double sum = 0; long cnt = 0;
    for (int k = P.k1; k <= P.k2; k++) for (int j = P.j1; j <= P.j2; j++) for (int i = P.i1; i <= P.i2; i++) {
      int i2 = i + (d == 0), j2 = j + (d == 1), k2 = k + (d == 2);
      if (i2 > P.i2 || j2 > P.j2 || k2 > P.k2) continue;
      size_t a = U(i,j,k), b = U(i2,j2,k2);
      double dx = (double)X[b]-X[a], dy = (double)Y[b]-Y[a], dz = (double)Z[b]-Z[a];
      sum += std::sqrt(dx*dx + dy*dy + dz*dz); cnt++;
    }
    float avg_dh = (float)(sum / cnt);
    float avg_L = avg_dh * P.L;
    int npt = P.L + 1;
    double Rpp = std::pow(10.0, -((std::log10((double)P.L) - 1.0) / std::log10(2.0) + 4.0));
    double dmax = -(double)c->pml_ref_vel[d][s] / (2.0 * avg_L) * std::log((float)Rpp) * 3.0;
    double amax = c->pml_alpha_max[d][s], bmax = c->pml_beta_max[d][s];
    P.A.assign(npt, 0.f); P.B.assign(npt, 0.f); P.D.assign(npt, 0.f);
    for (int n = 0; n < npt; n++) {
      double r = (double)(n * avg_dh) / avg_L;            // 0 at the interior edge, 1 outside
      double dd = dmax * r * r, aa = amax * (1.0 - r), bb = 1.0 + (bmax - 1.0) * r * r;
      int idx = s == 0 ? npt - 1 - n : n;
      P.D[idx] = (float)(dd / bb);                  // d / beta
      P.A[idx] = (float)(aa + dd / bb);             // alpha + d / beta
      P.B[idx] = (float)(1.0 / bb);                 // 1 / beta
    }
  }

  // ---- exponential sponge (bdry_ablexp_set, bdry_t.cu:453-700): six
  //      disjoint blocks (x slabs over all y and z, y slabs between them, z
  //      slabs inside both), each with the mask of its own direction; a
  //      point is scaled by the smallest of its three masks ------------------
  S.abl_nblk = 0;
  for (int d = 0; d < 3; d++) S.abl_E[d].assign(d == 0 ? nx : (d == 1 ? ny : nz), 1.f);
  {
    const int (&L)[3][2] = c->ablexp_layers;
    const int bx0 = ni1 + L[0][0], nbx = g.ni - L[0][0] - L[0][1];
    const int by0 = nj1 + L[1][0], nby = g.nj - L[1][0] - L[1][1];
    // [dim][side]: first index and count along each axis
    const int blk[6][6] = {
      { ni1, L[0][0], nj1, g.nj, nk1, g.nk }, { ni2 - L[0][1] + 1, L[0][1], nj1, g.nj, nk1, g.nk },
      { bx0, nbx, nj1, L[1][0], nk1, g.nk }, { bx0, nbx, nj2 - L[1][1] + 1, L[1][1], nk1, g.nk },
      { bx0, nbx, by0, nby, nk1, L[2][0] }, { bx0, nbx, by0, nby, nk2 - L[2][1] + 1, L[2][1] } };
    for (int n = 0; n < 6; n++) {
      const int d = n / 2, side = n % 2;
      const int *b = blk[n];
      if (c->ablexp_layers[d][side] <= 0 || b[1] <= 0 || b[3] <= 0 || b[5] <= 0) continue;
      const int lo[3] = { b[0], b[2], b[4] }, hi[3] = { b[0] + b[1] - 1, b[2] + b[3] - 1, b[4] + b[5] - 1 };
      // mean spacing along d (bdry_cal_abl_len_dh, bdry_t.cu:329-444): the
      // reference's loop order, summed in double
      const int a1 = d == 0 ? 2 : (d == 1 ? 2 : 1), a2 = d == 0 ? 1 : 0;   // outer, middle axes
      double sum = 0.0;
      long num = 0;
      int q[3];
      for (q[a1] = lo[a1]; q[a1] <= hi[a1]; q[a1]++)
        for (q[a2] = lo[a2]; q[a2] <= hi[a2]; q[a2]++) {
          q[d] = lo[d];
          size_t p0 = U(q[0], q[1], q[2]);
          double x0 = X[p0], y0 = Y[p0], z0 = Z[p0];
          for (q[d] = lo[d] + 1; q[d] <= hi[d]; q[d]++) {
            const size_t p1 = U(q[0], q[1], q[2]);
            const double x1 = X[p1], y1 = Y[p1], z1 = Z[p1];
            sum += std::sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0) + (z1 - z0) * (z1 - z0));
            x0 = x1; y0 = y1; z0 = z1;
            num += 1;
          }
        }
      const float dh = (float)(sum / num);
      const int nl = b[2 * d + 1];
      for (int m = lo[d]; m <= hi[d]; m++) {
        // the first layer inside the domain has the weakest damping
        const int layer = side == 0 ? nl - (m - lo[d]) : m - lo[d] + 1;
        S.abl_E[d][m] = ablexp_mask(layer, c->ablexp_ref_vel[d][side], c->dt, nl, dh);
      }
      int *o = S.abl_blk[S.abl_nblk++];
      o[0] = lo[0]; o[1] = hi[0]; o[2] = lo[1]; o[3] = hi[1]; o[4] = lo[2]; o[5] = hi[2];
    }
  }

  // ---- free surface conversion matrices (sv_curv_col_el_iso_dvh2dvz_gpu,
  //      sv_curv_col_el_iso_gpu.cu:1297-1405): at the top surface the
  //      traction-free condition A dV/dzeta = B dV/dxi + C dV/deta gives
  //      dV/dzeta = (A^-1 B) dV/dxi + (A^-1 C) dV/deta -----------------------
  S.free_mat.assign((size_t)2 * ny * nx * 9, 0.f);
  if (S.isfree) {
    for (int j = nj1; j <= nj2; j++) for (int i = ni1; i <= ni2; i++) {
      size_t p = U(i, j, nk2);
      double e1[3] = { Mp[MXIX][p], Mp[MXIY][p], Mp[MXIZ][p] };
      double e2[3] = { Mp[METX][p], Mp[METY][p], Mp[METZ][p] };
      double e3[3] = { Mp[MZTX][p], Mp[MZTY][p], Mp[MZTZ][p] };
      M3 A, B, Cm, Ai, AB, AC;
      dblock(e3, e3, lam[p], mu[p], 1.0, A);
      dblock(e3, e1, lam[p], mu[p], 1.0, B);
      dblock(e3, e2, lam[p], mu[p], 1.0, Cm);
      for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++) { B[r][q] = -B[r][q]; Cm[r][q] = -Cm[r][q]; }
      inv3(A, Ai); mul3(Ai, B, AB); mul3(Ai, Cm, AC);
      size_t o = ((size_t)j * nx + i) * 9;
      put9(AB, &S.free_mat[o]); put9(AC, &S.free_mat[(size_t)ny*nx*9 + o]);
    }
  }

  // ---- faults (fault_coef_cal + fault_set, fault_info.cu:98-1074) --------
  const size_t ns = (size_t)ny * nz;
  const int margin = c->welded_margin;
  for (int f = 0; f < c->num_faults; f++) {
    FaultHost Fh;
    Fh.i0 = c->fault_x_index[f] - 1 + NG;
    if (Fh.i0 < ni1 + 4 || Fh.i0 > ni2 - 4) { msg = "fault_x_index must be at least 5 points from the x sides"; return CGFD_ERR_ARG; }
    for (int q = 0; q < 4; q++) Fh.grid[q] = c->fault_grid[f][q] - 1;
    Fh.flag.assign(ns, 0);
    Fh.mat.assign((size_t)NFM * ns * 9, 0.f);
    Fh.fmat.assign((size_t)NFF * ny * 9, 0.f);
    Fh.scal.assign((size_t)NFS * ns, 0.f);
    Fh.out.assign((size_t)CGFD_FAULT_NFIELD * ns, 0.f);
    auto MAT = [&](int m, size_t node) { return &Fh.mat[((size_t)m * ns + node) * 9]; };
    auto FMT = [&](int m, int j) { return &Fh.fmat[((size_t)m * ny + j) * 9]; };
    auto SC = [&](int q, size_t node) -> float & { return Fh.scal[(size_t)q * ns + node]; };
    for (int k = 0; k < nz; k++) for (int j = 0; j < ny; j++) {
      size_t node = (size_t)j + (size_t)k * ny, p = U(Fh.i0, j, k);
      double e1[3] = { Mp[MXIX][p], Mp[MXIY][p], Mp[MXIZ][p] };
      double e2[3] = { Mp[METX][p], Mp[METY][p], Mp[METZ][p] };
      double e3[3] = { Mp[MZTX][p], Mp[MZTY][p], Mp[MZTZ][p] };
      const double *ea[3] = { e1, e2, e3 };
      double J = Mp[MJAC][p], la = lam[p], m_ = mu[p];
      M3 D[3][3];   // D[a][b], same medium on both sides
      for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) dblock(ea[a], ea[b], la, m_, J, D[a][b]);
      for (int side = 0; side < 2; side++)
        for (int a = 1; a < 3; a++) for (int b = 0; b < 3; b++)
          put9(D[a][b], MAT(side*6 + (a-1)*3 + b, node));
      M3 Dinv, t;
      inv3(D[0][0], Dinv);
      // method 1: split-node normal derivative of one side from the other
      mul3(Dinv, D[0][0], t); put9(t, MAT(FM_M2P1, node)); put9(t, MAT(FM_P2M1, node));
      mul3(Dinv, D[0][1], t); put9(t, MAT(FM_M2P2, node)); put9(t, MAT(FM_P2M2, node));
      put9(t, MAT(FM_M2P4, node)); put9(t, MAT(FM_P2M4, node));
      mul3(Dinv, D[0][2], t); put9(t, MAT(FM_M2P3, node)); put9(t, MAT(FM_P2M3, node));
      put9(t, MAT(FM_M2P5, node)); put9(t, MAT(FM_P2M5, node));
      // method 2: normal derivative from the traction rate
      put9(Dinv, MAT(FM_T1VXMIN, node)); put9(Dinv, MAT(FM_T1VXPLUS, node));
      mul3(Dinv, D[0][1], t); put9(t, MAT(FM_VYVXMIN, node)); put9(t, MAT(FM_VYVXPLUS, node));
      mul3(Dinv, D[0][2], t); put9(t, MAT(FM_VZVXMIN, node)); put9(t, MAT(FM_VZVXPLUS, node));
      // base vectors: n = e1/|e1|, s1 = (dx/deta)/|.|, s2 = n x s1
      M3 Em = { { e1[0], e1[1], e1[2] }, { e2[0], e2[1], e2[2] }, { e3[0], e3[1], e3[2] } }, Ei;
      inv3(Em, Ei);
      double xet[3] = { Ei[0][1], Ei[1][1], Ei[2][1] };
      double s1[3] = { xet[0]/nrm(xet), xet[1]/nrm(xet), xet[2]/nrm(xet) };
      double vn[3] = { e1[0]/nrm(e1), e1[1]/nrm(e1), e1[2]/nrm(e1) };
      double s2[3]; cross(vn, s1, s2);
      for (int q = 0; q < 3; q++) { SC(FS_S1X+q, node) = (float)s1[q]; SC(FS_S2X+q, node) = (float)s2[q]; }
      SC(FS_RHO0, node) = rho[p]; SC(FS_RHO1, node) = rho[p];
      if (k == nk2) {
        // free-surface rows (fault_info.cu:657-840): traction-free top plus
        // continuity on the fault; the along-strike constraint has weight 0
        M3 Ai, Bm, Cm, V2Z_x, V2Z_y;
        inv3(D[2][2], Ai);
        for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++) { Bm[r][q] = -D[2][0][r][q]; Cm[r][q] = -D[2][1][r][q]; }
        mul3(Ai, Bm, V2Z_x); mul3(Ai, Cm, V2Z_y);
        double u2[3]; cross(e1, xet, u2);
        double n2 = nrm(u2); for (int q = 0; q < 3; q++) u2[q] /= n2;
        double ne1 = nrm(e1);
        double h[3] = { dot(u2, e1)/ne1, dot(u2, e2)/ne1, dot(u2, e3)/ne1 };
        M3 Df[3];
        for (int b = 0; b < 3; b++) for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++)
          Df[b][r][q] = D[0][b][r][q] + m_ * h[b] * u2[r] * e1[q];
        M3 t1, t2, Vx, Vy;
        mul3(Df[2], V2Z_x, t1); mul3(Df[2], V2Z_y, t2);
        for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++) { Vx[r][q] = Df[0][r][q] + t1[r][q]; Vy[r][q] = Df[1][r][q] + t2[r][q]; }
        M3 Vxi, P1, P2, P3;
        inv3(Vx, Vxi);
        mul3(Vxi, Vx, P1); mul3(Vxi, Vy, P2); mul3(Vxi, Vy, P3);
        for (int side = 0; side < 2; side++) {
          put9(V2Z_x, FMT(side ? FF_VX2VZ2 : FF_VX2VZ1, j));
          put9(V2Z_y, FMT(side ? FF_VY2VZ2 : FF_VY2VZ1, j));
        }
        put9(P1, FMT(FF_P2M1, j)); put9(P2, FMT(FF_P2M2, j)); put9(P3, FMT(FF_P2M3, j));
        put9(P1, FMT(FF_M2P1, j)); put9(P2, FMT(FF_M2P2, j)); put9(P3, FMT(FF_M2P3, j));
        put9(Vxi, FMT(FF_T1VXMIN, j)); put9(P3, FMT(FF_VYVXMIN, j));
        put9(Vxi, FMT(FF_T1VXPLUS, j)); put9(P3, FMT(FF_VYVXPLUS, j));
      }
    }
    // inputs, masks and initial outputs for interior nodes
    const size_t fsz = (size_t)g.nj * g.nk;
    for (int k = 0; k < g.nk; k++) for (int j = 0; j < g.nj; j++) {
      size_t node = (size_t)(j+NG) + (size_t)(k+NG)*ny, src = f*fsz + (size_t)j + (size_t)k*g.nj;
      float T0[3] = { c->T0x[src], c->T0y[src], c->T0z[src] };
      SC(FS_T0X, node) = T0[0]; SC(FS_T0Y, node) = T0[1]; SC(FS_T0Z, node) = T0[2];
      SC(FS_MUS, node) = c->mu_s[src]; SC(FS_MUD, node) = c->mu_d[src];
      SC(FS_DC, node) = c->Dc[src]; SC(FS_C0, node) = c->C0[src];
      if (!(c->Dc[src] > 0.f)) { msg = "Dc must be positive"; return CGFD_ERR_ARG; }
      size_t p = U(Fh.i0, j+NG, k+NG);
      double e1[3] = { Mp[MXIX][p], Mp[MXIY][p], Mp[MXIZ][p] };
      double vn[3] = { e1[0]/nrm(e1), e1[1]/nrm(e1), e1[2]/nrm(e1) };
      double s1[3] = { SC(FS_S1X,node), SC(FS_S1Y,node), SC(FS_S1Z,node) };
      double s2[3] = { SC(FS_S2X,node), SC(FS_S2Y,node), SC(FS_S2Z,node) };
      double Td[3] = { T0[0], T0[1], T0[2] };
      Fh.out[(size_t)CGFD_FAULT_TN * ns + node] = (float)dot(Td, vn);
      Fh.out[(size_t)CGFD_FAULT_TS1 * ns + node] = (float)dot(Td, s1);
      Fh.out[(size_t)CGFD_FAULT_TS2 * ns + node] = (float)dot(Td, s2);
      Fh.out[(size_t)CGFD_FAULT_INIT_T0 * ns + node] = -9999.9f;
      const int *fg = Fh.grid;
      uint8_t fl = 0;
      bool welded = !(j >= margin && j < g.nj - margin && k >= margin && (S.isfree || k < g.nk - margin));
      if (!welded) fl |= FL_SPLIT;
      if (!(j <= fg[0]+3 || j >= fg[1]-3)) fl |= FL_RUPY;
      if (!(k <= fg[2]+3 || k >= fg[3]-3)) fl |= FL_RUPZ;
      if (j >= fg[0]+3 && j <= fg[1]-3 && k >= fg[2]+3 && k <= fg[3]-3) fl |= FL_GRID;
      Fh.flag[node] = fl;
    }
    S.faults.push_back(std::move(Fh));
  }
  for (size_t a = 0; a < S.faults.size(); a++)
    for (size_t b = a+1; b < S.faults.size(); b++)
      if (std::abs(S.faults[a].i0 - S.faults[b].i0) < 9) { msg = "faults must be at least 9 x points apart"; return CGFD_ERR_ARG; }

  // ---- stations (io_recv_read_locate, io_funcs.cu:25-309; fault stations
  //      io_fault_recv_read_locate, io_funcs.cu:2170-2309) -----------------
  S.max_rec = std::max(0, c->max_records);
  for (int n = 0; n < c->num_stations; n++) {
    float gx = c->station_ijk[3*n], gy = c->station_ijk[3*n+1], gz = c->station_ijk[3*n+2];
    int ix = (int)gx, iy = (int)gy, iz = (int)gz;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= g.ni || iy >= g.nj || iz >= g.nk) { msg = "station outside the grid"; return CGFD_ERR_ARG; }
    for (int q = 0; q < 8; q++)
      S.sta_idx.push_back(g.at(ix + NG + (q & 1), iy + NG + ((q >> 1) & 1), iz + NG + ((q >> 2) & 1)));
    S.sta_w.push_back(gx - ix); S.sta_w.push_back(gy - iy); S.sta_w.push_back(gz - iz);
  }
  for (int n = 0; n < c->num_fault_stations; n++) {
    int f = c->fault_station_fault[n];
    float gy = c->fault_station_jk[2*n], gz = c->fault_station_jk[2*n+1];
    int iy = (int)std::floor(gy), iz = (int)std::floor(gz);
    if (f < 0 || f >= c->num_faults || iy < 0 || iz < 0 || iy >= g.nj || iz >= g.nk) { msg = "fault station outside the fault plane"; return CGFD_ERR_ARG; }
    S.fsta_fid.push_back(f);
    int J = iy + NG, K = iz + NG;
    S.fsta_idx.push_back(J + K*ny); S.fsta_idx.push_back(J+1 + K*ny);
    S.fsta_idx.push_back(J + (K+1)*ny); S.fsta_idx.push_back(J+1 + (K+1)*ny);
    S.fsta_w.push_back(gy - iy); S.fsta_w.push_back(gz - iz);
  }
  return CGFD_OK;
}

}  // namespace cgfd
