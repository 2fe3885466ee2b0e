// common.h -- data layout and device argument blocks shared by the host
// set-up (setup.cpp), the kernels (volume.cu, fault.cu) and the C ABI
// (api.cu).
//
// HBM layout.  Every 3-D field is stored like the reference's (3 ghost
// points per side, x fastest, src/forward/gd_t.cu:2124-2140) but with a
// padded row pitch: index p = (i + xoff) + j*sy + k*sz for ghost-inclusive
// indices (i, j, k), sy a multiple of 32 points.  xoff (0..7, per grid)
// puts the first point of the interior box (the first x index after the
// left PML) on a 128-byte line of the 16-byte component groups, so that a
// warp's 32 points of one row read exactly four lines.  A wavefield level holds the
// 9 components (Vx,Vy,Vz,Txx,Tyy,Tzz,Tyz,Txz,Txy) of scmp points as two
// arrays of 16-byte groups (Vx Vy Vz Txx | Tyy Tzz Tyz Txz) and one of Txy,
// so that a stencil tap reads all nine with three loads (Grid::w); four levels
// P (time n), A and B (ping-pong stage inputs) and E (time n+1 accumulator)
// replace the reference's pre/tmp/rhs/end, because each fused stage writes
// its output level directly instead of a separate rhs array.
#pragma once
#include <cstddef>
#include <cstdint>

#include "real.h"

#ifdef __CUDACC__
#define CGFD_HD __host__ __device__
#else
#define CGFD_HD
#endif

namespace cgfd {

constexpr int NG = 3;            // ghost points per side
constexpr int NCMP = 9;
constexpr int MAXF = 8;          // faults

enum Cmp { VX = 0, VY, VZ, TXX, TYY, TZZ, TYZ, TXZ, TXY };
// fault wavefield components [side][comp] (src/forward/fault_wav_t.cu:96-150)
enum FCmp { FVX = 0, FVY, FVZ, FT2X, FT2Y, FT2Z, FT3X, FT3Y, FT3Z };
// metric component order in the host metric block
enum Met { MJAC = 0, MXIX, MXIY, MXIZ, METX, METY, METZ, MZTX, MZTY, MZTZ };
// On the device the metric and the medium are one block of 13 scmp floats:
// the Jacobian plane, then three arrays of 16-byte groups, one per
// contravariant direction d, each holding that direction's metric row and
// one medium value: (xi_x xi_y xi_z lambda), (eta_x eta_y eta_z mu),
// (zeta_x zeta_y zeta_z 1/rho).
#ifdef __CUDACC__
__device__ __forceinline__ real4 coef_row(const real *cf, long scmp, int d, long q) {
  return __ldg(reinterpret_cast<const real4 *>(cf + scmp) + d * scmp + q);
}
__device__ __forceinline__ real coef_jac(const real *cf, long q) { return __ldg(cf + q); }
#endif

// per-node 3x3 fault matrices, [NFM][nodes][9]
enum FaultMat {
  FM_D21_1 = 0, FM_D22_1, FM_D23_1, FM_D31_1, FM_D32_1, FM_D33_1,
  FM_D21_2, FM_D22_2, FM_D23_2, FM_D31_2, FM_D32_2, FM_D33_2,
  FM_M2P1, FM_M2P2, FM_M2P3, FM_M2P4, FM_M2P5,
  FM_P2M1, FM_P2M2, FM_P2M3, FM_P2M4, FM_P2M5,
  FM_T1VXMIN, FM_VYVXMIN, FM_VZVXMIN, FM_T1VXPLUS, FM_VYVXPLUS, FM_VZVXPLUS,
  NFM
};
// per-strike-column free-surface fault matrices, [NFF][ny][9]
enum FaultFreeMat {
  FF_VX2VZ1 = 0, FF_VY2VZ1, FF_VX2VZ2, FF_VY2VZ2,
  FF_P2M1, FF_P2M2, FF_P2M3, FF_M2P1, FF_M2P2, FF_M2P3,
  FF_T1VXMIN, FF_VYVXMIN, FF_T1VXPLUS, FF_VYVXPLUS,
  NFF
};
// per-node scalar fault data, [NFS][nodes]
enum FaultScal {
  FS_T0X = 0, FS_T0Y, FS_T0Z, FS_MUS, FS_MUD, FS_DC, FS_C0,
  FS_RHO0, FS_RHO1,                 // rho on the minus / plus side
  FS_S1X, FS_S1Y, FS_S1Z, FS_S2X, FS_S2Y, FS_S2Z,
  FS_TTN, FS_TTS1, FS_TTS2,         // stage traction (not stored; kept for layout)
  FS_T1X, FS_T1Y, FS_T1Z,           // traction at the split node of this stage
  FS_HT1X, FS_HT1Y, FS_HT1Z,        // dT1/dt of the last step
  FS_MT1X, FS_MT1Y, FS_MT1Z,        // T1 of the last step
  NFS
};
// fault node flags (uint8 bits)
enum FaultFlag { FL_SPLIT = 1, FL_RUPY = 2, FL_RUPZ = 4, FL_GRID = 8, FL_T0SET = 16, FL_RUP = 32 };

struct Grid {
  int ni, nj, nk;        // interior points
  int nx, ny, nz;        // with ghosts
  int xoff;              // x offset of the row pitch (see above)
  long sy, sz;           // strides of j and k (elements)
  long scmp;             // elements per component (sz * nz)
  CGFD_HD long at(int i, int j, int k) const { return (long)(i + xoff) + (long)j * sy + (long)k * sz; }
  // element of component c at point p within one wavefield level: the
  // components 0-3 (Vx Vy Vz Txx) and 4-7 (Tyy Tzz Tyz Txz) are interleaved
  // in 16-byte groups, Txy is stored alone
  CGFD_HD long w(int c, long p) const { return c < 4 ? 4 * p + c : (c < 8 ? 4 * scmp + 4 * p + (c - 4) : 8 * scmp + p); }
};
// distance between neighbouring points of one wavefield component (floats)
CGFD_HD constexpr int wstep(int c) { return c < 8 ? 4 : 1; }

struct PmlFaceDev {
  int on, d, s, L;
  int i1, j1, k1;        // first point of the face region (ghost-inclusive indices)
  int fni, fnj, fnk;     // face region extents
  long siz;              // fni*fnj*fnk
  const real *A, *B, *D;   // per layer along the normal
  // auxiliary-field levels used by one stage (9*siz floats each, grouped
  // like a wavefield level with siz points per component): stage input,
  // time-n level, next-stage output, end accumulator
  const real *acur, *apre;
  real *aout, *aend;
};

struct FaultDev {
  int i0;                   // ghost-inclusive x index of the fault plane
  int bit;
  const uint8_t *flag_in;   // FL_SPLIT / FL_RUPY / FL_RUPZ / FL_GRID per node [ny*nz]
  uint8_t *flag;            // mutable flags (FL_T0SET, FL_RUP)
  const real *mat;         // [NFM][ny*nz][9]
  const real *fmat;        // [NFF][ny][9]
  real *scal;              // [NFS][ny*nz]
  real *out;               // [11][ny*nz] Tn..Init_t0
};

struct StationDev {
  int n, nf, max_rec;
  const long *idx;          // [n][8] volume indices (corner 4 unused: reference quirk)
  const real *w;           // [n][3] di, dj, dk
  const int *fid;           // [nf] fault id
  const int *fidx;          // [nf][4] node indices
  const real *fw;          // [nf][2] dj, dk
  real *seis;              // [n][9][max_rec]
  real *fseis;             // [nf][9][max_rec]
};

// control block in device memory, advanced on the device so that a step
// can be replayed as a CUDA graph
struct Ctl {
  int it;                   // steps taken
  int nrec;                 // records taken
  int err;                  // CTL_ERR_* bits
  int pad;
};
enum CtlErr { CTL_ERR_NONFINITE = 1 };

}  // namespace cgfd
