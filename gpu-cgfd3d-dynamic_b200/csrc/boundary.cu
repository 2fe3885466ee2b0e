// boundary.cu -- end-of-step work on the level of time n+1, after the last
// RK stage (drv_rk_curv_col.cu:596-612):
//   * exponential sponge   bdry_ablexp_apply_gpu (src/forward/bdry_t.cu:764-818)
//   * surface peak motion  PG_calcu_gpu (src/forward/wav_t.cu:138-216)
// Both are HBM-bound passes over a subset of the grid: the sponge reads and
// writes the nine components of its layers (72 B per point), the peaks
// read six velocities and read-modify-write 18 surface values per surface
// point.
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

// one thread per sponge point, x fastest within each block
__global__ void __launch_bounds__(256) k_sponge(const SpongeArgs a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.first[a.nblk]) return;
  int b = 0;
  while (b + 1 < a.nblk && t >= a.first[b + 1]) b++;
  const int *B = a.blk[b];
  const long u = t - a.first[b];
  const int ni = B[1] - B[0] + 1, nj = B[3] - B[2] + 1;
  const int i = B[0] + (int)(u % ni), j = B[2] + (int)((u / ni) % nj), k = B[4] + (int)(u / ((long)ni * nj));
  const Grid &g = a.g;
  const real ex = __ldg(a.E + i), ey = __ldg(a.E + g.nx + j), ez = __ldg(a.E + g.nx + g.ny + k);
  // the reference's selection order: min(Ex, Ey), then Ez
  real mask = ex < ey ? ex : ey;
  if (mask > ez) mask = ez;
  const long p = g.at(i, j, k), sc = g.scmp;
  real4 *A = reinterpret_cast<real4 *>(a.w) + p, *Bq = reinterpret_cast<real4 *>(a.w + 4 * sc) + p;
  real4 x = *A, y = *Bq;
  real tz = a.w[8 * sc + p];
  x.x *= mask; x.y *= mask; x.z *= mask; x.w *= mask;
  y.x *= mask; y.y *= mask; y.z *= mask; y.w *= mask;
  *A = x; *Bq = y;
  a.w[8 * sc + p] = tz * mask;
}

// one thread per surface point (interior i, j) at the top row
__global__ void __launch_bounds__(256) k_surface_peaks(const PeakArgs a) {
  const Grid &g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.ni || j >= g.nj) return;
  const long p = g.at(i + NG, j + NG, g.nk + NG - 1);
  // velocities are the first three lanes of the first 16-byte group
  const real4 v1 = __ldg(reinterpret_cast<const real4 *>(a.wend) + p);
  const real4 v0 = __ldg(reinterpret_cast<const real4 *>(a.wpre) + p);
  const long n = (long)g.ni * g.nj, q = i + (long)j * g.ni;
  const real dt = a.dt;
  const real Ax = fabs((v1.x - v0.x) / dt), Ay = fabs((v1.y - v0.y) / dt), Az = fabs((v1.z - v0.z) / dt);
  // displacement by the trapezoid rule, accumulated through double as in
  // the reference (its 0.5 is a double constant)
  real Dx = a.dis[q], Dy = a.dis[n + q], Dz = a.dis[2 * n + q];
  Dx += 0.5 * (v1.x + v0.x) * dt;
  Dy += 0.5 * (v1.y + v0.y) * dt;
  Dz += 0.5 * (v1.z + v0.z) * dt;
  a.dis[q] = Dx; a.dis[n + q] = Dy; a.dis[2 * n + q] = Dz;
  const real val[15] = {
      sqrt(v1.x * v1.x + v1.y * v1.y + v1.z * v1.z), sqrt(v1.x * v1.x + v1.y * v1.y),
      fabs(v1.x), fabs(v1.y), fabs(v1.z),
      sqrt(Ax * Ax + Ay * Ay + Az * Az), sqrt(Ax * Ax + Ay * Ay), Ax, Ay, Az,
      sqrt(Dx * Dx + Dy * Dy + Dz * Dz), sqrt(Dx * Dx + Dy * Dy), fabs(Dx), fabs(Dy), fabs(Dz) };
#pragma unroll
  for (int c = 0; c < 15; c++) {
    real *o = a.pg + c * n + q;
    if (*o < val[c]) *o = val[c];
  }
}

}  // namespace

int launch_sponge(const SpongeArgs &a, cudaStream_t st) {
  const long n = a.first[a.nblk];
  if (n <= 0) return 0;
  k_sponge<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
  return 1;
}

int launch_surface_peaks(const PeakArgs &a, cudaStream_t st) {
  const dim3 blk(32, 8);
  const dim3 grd((a.g.ni + 31) / 32, (a.g.nj + 7) / 8);
  k_surface_peaks<<<grd, blk, 0, st>>>(a);
  return 1;
}

}  // namespace cgfd
