// setup.h -- host set-up of one forward problem (grid, metric, medium,
// stability limit, CFS-PML profiles, free-surface matrices, fault
// coefficients and masks, station indices), producing arrays in the device
// layout of common.h.  Restates the set-up half of the reference's main
// (src/forward/main_curv_col_el_3d.cu:113-705); computed in double and
// stored as float.
#pragma once
#include <string>
#include <vector>

#include "../../include/cgfd.h"
#include "common.h"

namespace cgfd {

struct PmlHost {
  int on = 0, L = 0;
  int i1, i2, j1, j2, k1, k2;
  std::vector<float> A, B, D;
};

struct FaultHost {
  int i0 = 0;
  int grid[4];                    // 0-based j1, j2, k1, k2
  std::vector<uint8_t> flag;      // [ny*nz]
  std::vector<float> mat;         // [NFM][ny*nz][9]
  std::vector<float> fmat;        // [NFF][ny][9]
  std::vector<float> scal;        // [NFS][ny*nz]
  std::vector<float> out;         // [11][ny*nz]
};

struct HostSetup {
  Grid g;
  float dt = 0.f, dtmax = 0.f;
  int imethod = 2, isfree = 0;
  // metric and medium as the device reads them: [scmp] Jacobian, then
  // [3][scmp][4] (metric row d, medium value d) with the medium values
  // lambda, mu, 1/rho
  std::vector<float> coef;
  std::vector<float> free_mat;    // [2][ny][nx][9]: matVx2Vz, matVy2Vz at the surface
  std::vector<float> coords;      // [3][nk][nj][ni]: x, y, z of the interior grid points
  PmlHost pml[3][2];
  // exponential sponge: masks along x, y, z (ghost-inclusive index, 1 outside
  // the layers) and the blocks they scale (ghost-inclusive, inclusive bounds
  // i1 i2 j1 j2 k1 k2)
  int abl_nblk = 0;
  int abl_blk[6][6];
  std::vector<float> abl_E[3];
  std::vector<FaultHost> faults;
  // stations
  std::vector<long> sta_idx;      // [n][8]
  std::vector<float> sta_w;       // [n][3]
  std::vector<int> fsta_fid;      // [nf]
  std::vector<int> fsta_idx;      // [nf][4]
  std::vector<float> fsta_w;      // [nf][2]
  int max_rec = 0;
};

// Returns CGFD_OK or a CGFD_ERR_* code; msg receives the reason.
int build_setup(const cgfd_config *c, HostSetup &S, std::string &msg);

}  // namespace cgfd
