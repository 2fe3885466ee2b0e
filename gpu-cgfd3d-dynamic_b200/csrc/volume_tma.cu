// volume_tma.cu -- TMA-fed, z-marching volume stage kernel for sm_100a.
//
// The operator is the reference's inner volume RHS + CFS-PML correction +
// RK stage update (sv_curv_col_el_iso_gpu.cu:232-388 and :825-1290,
// wav_t.cu:219-234, drv_rk_curv_col.cu:329-568) for every row below the
// four rows under the free surface (those run k_volume<SHELL> in
// volume.cu, which adds the traction image and velocity-low operators).
// Data movement:
//   * a block owns 32 (x) x 8 (y) columns and marches a chunk of z rows;
//   * the stage's input level is read only through TMA: one
//     cp.async.bulk.tensor.4d per z row brings the 9 components of a
//     40 x 14 tile (x halo rounded out to 16-byte boundaries, y halo 3+3)
//     into a ring of five row buffers in shared memory, completion tracked
//     by one mbarrier per buffer; loads run two rows ahead of the compute;
//   * x / y derivatives read the current row's buffer, z derivatives a
//     per-thread register queue of five samples fed from the ring;
//   * metric, medium, the time-n level and the end accumulator are read
//     point-wise (coalesced) before the row wait, so their latency overlaps
//     it; outputs are written point-wise;
//   * the RHS accumulates each derivative straight into the velocity
//     gradient and the momentum sums; a point in a CFS-PML face recomputes
//     direction d's part from the staged row (or the queue) afterwards.
// The row loop is unrolled five-fold so the queue never moves: logical slot
// m of row phase PH lives in register q[.][(m + PH) % 5].
// Waits on an mbarrier are bounded: after the limit the kernel records
// CTL_ERR_TMA in the control block and stops working on its rows.
#include <cuda.h>
#include <cuda_runtime.h>

#include "ops.cuh"

namespace cgfd {

namespace {

constexpr int TX = 32, TY = 8;
constexpr int BOXX = 40, BOXY = 14;           // TMA box: x from 32*bx (aligned), y from 8*by
constexpr int XC = 4, YC = 3;                 // tile position of the block's first own point
constexpr int NBUF = 5;
constexpr int PLANE = 9 * BOXY * BOXX;        // floats per row buffer
constexpr int PLANE_BYTES = PLANE * 4;        // 20160
constexpr int PLANE_STRIDE = (PLANE_BYTES + 127) / 128 * 128;
constexpr unsigned WAIT_LIMIT = 1u << 26;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// bounded wait; false if the limit was hit
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned limit = WAIT_LIMIT) {
  for (unsigned n = 0; n < limit; n++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, uint64_t *bar, int x, int y, int z, int c) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
      ::"r"(smem_addr(dst)), "l"(tm), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_addr(bar))
      : "memory");
}

template <int F>
__device__ __forceinline__ float wdrp(int n) {
  return F ? (n == 0 ? kC1 : n == 1 ? kC2 : n == 2 ? kC3 : n == 3 ? kC4 : kC5)
           : (n == 0 ? -kC5 : n == 1 ? -kC4 : n == 2 ? -kC3 : n == 3 ? -kC2 : -kC1);
}

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

// PML face P (normal d) at this point: correction from direction d's part
// of the RHS (recomputed from the staged tile / queue), aux-field update
template <int MODE>
__device__ __forceinline__ void pml_face(const VolArgs &a, const PmlFaceDev &P, int d, int I, int J, int K,
                                         const float r[9], float corr[9]) {
  const int li = I - P.i1, lj = J - P.j1, lk = K - P.k1;
  if (li < 0 || li >= P.fni || lj < 0 || lj >= P.fnj || lk < 0 || lk >= P.fnk) return;
  const int layer = d == 0 ? li : (d == 1 ? lj : lk);
  const float cA = __ldg(P.A + layer), cB = __ldg(P.B + layer), cD = __ldg(P.D + layer);
  const long pa = li + (long)lj * P.fni + (long)lk * P.fni * P.fnj;
#pragma unroll
  for (int c = 0; c < 9; c++) {
    const long o = c * P.siz + pa;
    const float av = __ldg(P.acur + o);
    corr[c] += (cB - 1.0f) * r[c] - cB * av;
    const float ar = cD * r[c] - cA * av;
    if (MODE == RK_FIRST) {
      P.aout[o] = av + a.ca * ar;
      P.aend[o] = av + a.cb * ar;
    } else if (MODE == RK_MID) {
      P.aout[o] = __ldg(P.apre + o) + a.ca * ar;
      P.aend[o] += a.cb * ar;
    } else {
      P.aend[o] += a.cb * ar;
    }
  }
}

struct RowCtx {
  const float *tile0;         // ring base (shared memory)
  uint64_t *bar;
  int tx, ty, tid, I, J, kb, K0, Klast, tmx, tmy;
  bool inside, colpml;
  int slab_f;
  long sc;
};

// one z row of the march; PH = row index mod 5 selects the queue rotation
// (logical queue slot m lives in q[.][(m + PH) % 5]) so that no values move
template <int ID, int JD, int KD, int MODE, int PH>
__device__ __forceinline__ bool row_step(const CUtensorMap &tm, const VolArgs &a, const RowCtx &x,
                                         float (&q)[9][5], int k, bool &alive) {
  constexpr int ZF = KD ? 3 : 1;
  constexpr int M0 = KD ? 1 : 3;
  const Grid &g = a.g;
  const long sc = x.sc;
  const int K = k + NG, r = k - x.kb;
  const long p = g.at(x.I, x.J, K);
  bool work = x.inside;
  if (work && x.slab_f >= 0 && (__ldg(a.fflag[x.slab_f] + x.J + (long)K * g.ny) & FL_SPLIT)) work = false;
  // metric and medium first, so their latency overlaps the row wait
  float e[9], lam = 0.f, mu = 0.f, slw = 0.f;
  if (work) {
#pragma unroll
    for (int c = 0; c < 9; c++) e[c] = __ldg(a.met + (1 + c) * sc + p);
    lam = __ldg(a.med + p); mu = __ldg(a.med + sc + p); slw = __ldg(a.med + 2 * sc + p);
  }
  const int sR = r % NBUF, sF = (r + ZF) % NBUF;
  const bool mine = mbar_wait(&x.bar[sR], (r / NBUF) & 1) && mbar_wait(&x.bar[sF], ((r + ZF) / NBUF) & 1);
  if (__syncthreads_and(mine) == 0) { alive = false; return false; }
  const float *tR = x.tile0 + sR * (PLANE_STRIDE / 4);
  const float *tF = x.tile0 + sF * (PLANE_STRIDE / 4);
  const int own = (YC + x.ty) * BOXX + XC + x.tx;
#pragma unroll
  for (int c = 0; c < 9; c++) q[c][(4 + PH) % 5] = tF[c * BOXY * BOXX + own];

  if (work) {
    const float l2m = lam + 2.0f * mu;
    float G[3][3] = { { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f }, { 0.f, 0.f, 0.f } };
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    // x and y from the staged row, z from the queue; each derivative goes
    // straight into the velocity gradient / momentum sums
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      const float *ea = e + 3 * dir;
#pragma unroll
      for (int c = 0; c < 9; c++) {
        float d = 0.f;
        if (dir == 0) {
          const float *row = tR + c * BOXY * BOXX + own;
#pragma unroll
          for (int n = 0; n < 5; n++) d += wdrp<ID>(n) * row[ID ? n - 1 : n - 3];
        } else if (dir == 1) {
          const float *col = tR + c * BOXY * BOXX + own;
#pragma unroll
          for (int n = 0; n < 5; n++) d += wdrp<JD>(n) * col[(JD ? n - 1 : n - 3) * BOXX];
        } else {
#pragma unroll
          for (int n = 0; n < 5; n++) d += wdrp<KD>(n) * q[c][(n + PH) % 5];
        }
        if (c < 3) { G[c][0] += ea[0] * d; G[c][1] += ea[1] * d; G[c][2] += ea[2] * d; }
        else if (c == TXX) s0 += ea[0] * d;
        else if (c == TYY) s1 += ea[1] * d;
        else if (c == TZZ) s2 += ea[2] * d;
        else if (c == TYZ) { s1 += ea[2] * d; s2 += ea[1] * d; }
        else if (c == TXZ) { s0 += ea[2] * d; s2 += ea[0] * d; }
        else { s0 += ea[1] * d; s1 += ea[0] * d; }
      }
    }
    float h[9];
    h[VX] = slw * s0; h[VY] = slw * s1; h[VZ] = slw * s2;
    h[TXX] = l2m * G[0][0] + lam * (G[1][1] + G[2][2]);
    h[TYY] = l2m * G[1][1] + lam * (G[0][0] + G[2][2]);
    h[TZZ] = l2m * G[2][2] + lam * (G[0][0] + G[1][1]);
    h[TXY] = mu * (G[0][1] + G[1][0]);
    h[TXZ] = mu * (G[0][2] + G[2][0]);
    h[TYZ] = mu * (G[1][2] + G[2][1]);
    const bool rowpml = (a.pml[4].on && K <= a.pml[4].k1 + a.pml[4].fnk - 1) || (a.pml[5].on && K >= a.pml[5].k1);
    if (x.colpml || rowpml) {
      // CFS-PML: each face adds (B-1) r_d - B aux from direction d's part
      float corr[9];
#pragma unroll
      for (int c = 0; c < 9; c++) corr[c] = 0.f;
#pragma unroll
      for (int fc = 0; fc < 6; fc++) {
        const int d = fc >> 1;
        if (!a.pml[fc].on) continue;
        const PmlFaceDev &P = a.pml[fc];
        const int li = x.I - P.i1, lj = x.J - P.j1, lk = K - P.k1;
        if (li < 0 || li >= P.fni || lj < 0 || lj >= P.fnj || lk < 0 || lk >= P.fnk) continue;
        float D[9], rr[9];
#pragma unroll
        for (int c = 0; c < 9; c++) {
          float dd = 0.f;
          if (d == 0) {
            const float *row = tR + c * BOXY * BOXX + own;
#pragma unroll
            for (int n = 0; n < 5; n++) dd += wdrp<ID>(n) * row[ID ? n - 1 : n - 3];
          } else if (d == 1) {
            const float *col = tR + c * BOXY * BOXX + own;
#pragma unroll
            for (int n = 0; n < 5; n++) dd += wdrp<JD>(n) * col[(JD ? n - 1 : n - 3) * BOXX];
          } else {
#pragma unroll
            for (int n = 0; n < 5; n++) dd += wdrp<KD>(n) * q[c][(n + PH) % 5];
          }
          D[c] = dd;
        }
        rhs_dir(D, e + 3 * d, lam, mu, l2m, slw, rr);
        pml_face<MODE>(a, P, d, x.I, x.J, K, rr, corr);
      }
#pragma unroll
      for (int c = 0; c < 9; c++) h[c] += corr[c];
    }
#pragma unroll
    for (int c = 0; c < 9; c++) {
      const long o = c * sc + p;
      if (MODE == RK_FIRST) {
        const float v = q[c][(M0 + PH) % 5];
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
  // row buffer sR is free once every thread is past this row
  __syncthreads();
  if (K + NBUF <= x.Klast && x.tid == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&x.bar[sR], PLANE_BYTES);
    tma_load_4d((void *)(x.tile0 + sR * (PLANE_STRIDE / 4)), &tm, &x.bar[sR], x.tmx, x.tmy, K + NBUF, 0);
  }
  return true;
}

template <int ID, int JD, int KD, int MODE>
__global__ void __launch_bounds__(TX * TY, 2)
    k_volume_tma(const __grid_constant__ CUtensorMap tm, const __grid_constant__ VolArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + NBUF * PLANE_STRIDE);
  constexpr int ZF = KD ? 3 : 1;

  const Grid &g = a.g;
  RowCtx x;
  x.sc = g.scmp;
  x.tx = threadIdx.x; x.ty = threadIdx.y; x.tid = x.ty * TX + x.tx;
  const int i = blockIdx.x * TX + x.tx, j = blockIdx.y * TY + x.ty;
  x.I = i + NG; x.J = j + NG;
  x.inside = i < g.ni && j < g.nj;
  const bool valid = x.I < g.nx && x.J < g.ny;
  x.kb = blockIdx.z * a.kchunk;
  const int ke = min(x.kb + a.kchunk, a.kend);
  if (x.kb >= ke) return;
  x.K0 = x.kb + NG; x.Klast = ke - 1 + NG + ZF;
  x.tmx = blockIdx.x * TX; x.tmy = blockIdx.y * TY;
  x.tile0 = reinterpret_cast<const float *>(smem);
  x.bar = bar;
  x.colpml = false;
#pragma unroll
  for (int fc = 0; fc < 4; fc++) {
    const PmlFaceDev &P = a.pml[fc];
    if (P.on && x.I >= P.i1 && x.I < P.i1 + P.fni && x.J >= P.j1 && x.J < P.j1 + P.fnj) x.colpml = true;
  }
  x.slab_f = -1;
  for (int f = 0; f < a.nfault; f++) {
    const int d = x.I - a.fi0[f];
    if (d >= -3 && d <= 3) x.slab_f = f;
  }

  if (x.tid == 0) {
    for (int s = 0; s < NBUF; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (x.tid == 0) {
    for (int s = 0; s < NBUF && x.K0 + s <= x.Klast; s++) {
      mbar_expect_tx(&bar[s], PLANE_BYTES);
      tma_load_4d(smem + s * PLANE_STRIDE, &tm, &bar[s], x.tmx, x.tmy, x.K0 + s, 0);
    }
  }
  // z queue, logical slots 0..3 = rows K0 + (KD ? m-1 : m-3)
  float q[9][5];
  {
    const long p0 = valid ? g.at(x.I, x.J, x.K0) : 0;
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const long o = p0 + (long)(KD ? m - 1 : m - 3) * g.sz;
#pragma unroll
      for (int c = 0; c < 9; c++) q[c][m] = valid ? __ldg(a.cur + c * x.sc + o) : 0.f;
    }
  }
  bool alive = true;
  int k = x.kb;
  for (; k + 5 <= ke; k += 5) {
    if (!row_step<ID, JD, KD, MODE, 0>(tm, a, x, q, k, alive)) break;
    if (!row_step<ID, JD, KD, MODE, 1>(tm, a, x, q, k + 1, alive)) break;
    if (!row_step<ID, JD, KD, MODE, 2>(tm, a, x, q, k + 2, alive)) break;
    if (!row_step<ID, JD, KD, MODE, 3>(tm, a, x, q, k + 3, alive)) break;
    if (!row_step<ID, JD, KD, MODE, 4>(tm, a, x, q, k + 4, alive)) break;
  }
  if (alive && k < ke) {
    const int left = ke - k;
    if (row_step<ID, JD, KD, MODE, 0>(tm, a, x, q, k, alive) && left > 1 &&
        row_step<ID, JD, KD, MODE, 1>(tm, a, x, q, k + 1, alive) && left > 2 &&
        row_step<ID, JD, KD, MODE, 2>(tm, a, x, q, k + 2, alive) && left > 3)
      row_step<ID, JD, KD, MODE, 3>(tm, a, x, q, k + 3, alive);
  }
  if (!alive && x.tid == 0) {
    // a row buffer did not arrive in time: flag it, then give the copies
    // still in flight a bounded chance to land before the block's shared
    // memory is released
    atomicOr(a.ctl_err, CTL_ERR_TMA);
    for (int s = 0; s < NBUF; s++) {
      mbar_wait(&bar[s], 0, 1u << 14);
      mbar_wait(&bar[s], 1, 1u << 14);
    }
  }
}

template <int ID, int JD, int KD, int MODE>
void prep_one() {
  cudaFuncSetAttribute(k_volume_tma<ID, JD, KD, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       NBUF * PLANE_STRIDE + NBUF * 8);
}
template <int ID, int JD, int KD>
void prep3() { prep_one<ID, JD, KD, RK_FIRST>(); prep_one<ID, JD, KD, RK_MID>(); prep_one<ID, JD, KD, RK_LAST>(); }

template <int ID, int JD, int KD>
void launch_m(const CUtensorMap &tm, const VolArgs &a, int mode, cudaStream_t st) {
  const dim3 blk(TX, TY, 1);
  const dim3 grd((a.g.ni + TX - 1) / TX, (a.g.nj + TY - 1) / TY, (a.g.nk + a.kchunk - 1) / a.kchunk);
  const size_t shm = NBUF * PLANE_STRIDE + NBUF * 8;
  if (mode == RK_FIRST) k_volume_tma<ID, JD, KD, RK_FIRST><<<grd, blk, shm, st>>>(tm, a);
  else if (mode == RK_MID) k_volume_tma<ID, JD, KD, RK_MID><<<grd, blk, shm, st>>>(tm, a);
  else k_volume_tma<ID, JD, KD, RK_LAST><<<grd, blk, shm, st>>>(tm, a);
}

}  // namespace

// shared-memory opt-in of every instantiation (once, before any capture)
void volume_tma_prepare() {
  prep3<0, 0, 0>(); prep3<0, 0, 1>(); prep3<0, 1, 0>(); prep3<0, 1, 1>();
  prep3<1, 0, 0>(); prep3<1, 0, 1>(); prep3<1, 1, 0>(); prep3<1, 1, 1>();
}

// 4-D tensor map (x, y, z, component) over one wavefield level; the box is
// the 40 x 14 x 1 x 9 row tile
int volume_tma_encode(CUtensorMap *tm, const float *level, const Grid &g) {
  typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                               const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return -1;
    fn = (EncodeFn)p;
  }
  const cuuint64_t dims[4] = { (cuuint64_t)g.sy, (cuuint64_t)g.ny, (cuuint64_t)g.nz, 9 };
  const cuuint64_t strides[3] = { (cuuint64_t)g.sy * 4, (cuuint64_t)g.sz * 4, (cuuint64_t)g.scmp * 4 };
  const cuuint32_t box[4] = { BOXX, BOXY, 1, 9 };
  const cuuint32_t estr[4] = { 1, 1, 1, 1 };
  CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)level, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -2;
}

void launch_volume_tma(const CUtensorMap &tm, const VolArgs &a, int idir, int jdir, int kdir, int mode,
                       cudaStream_t st) {
  switch (idir * 4 + jdir * 2 + kdir) {
    case 0: launch_m<0, 0, 0>(tm, a, mode, st); break;
    case 1: launch_m<0, 0, 1>(tm, a, mode, st); break;
    case 2: launch_m<0, 1, 0>(tm, a, mode, st); break;
    case 3: launch_m<0, 1, 1>(tm, a, mode, st); break;
    case 4: launch_m<1, 0, 0>(tm, a, mode, st); break;
    case 5: launch_m<1, 0, 1>(tm, a, mode, st); break;
    case 6: launch_m<1, 1, 0>(tm, a, mode, st); break;
    default: launch_m<1, 1, 1>(tm, a, mode, st); break;
  }
}

}  // namespace cgfd
