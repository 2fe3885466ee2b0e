// api.cu -- the C ABI of include/cgfd.h.
//
// cgfd_create runs the host set-up (setup.cpp), allocates the device state
// and copies the problem once.  cgfd_run replays one CUDA graph per time
// step; there are eight graphs, one per MacCormack operator pair
// (it % 8, src/forward/drv_rk_curv_col.cu:237), each holding the station
// sample, 4 x (fault-plane kernels + fused volume kernel) and the step
// counter advance.  Time levels P and E swap by step parity, which it % 8
// fixes, so the graphs never need their arguments updated.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdlib>
#include <map>
#include <mutex>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cgfd.h"
#include "ops.cuh"
#include "setup.h"

namespace cgfd {
void volume_boxes(VolArgs &a, const int (*boxes)[6], int n, bool pack);
void launch_volume_interior(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_shell(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_face_x(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_face_y(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_face_z(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_edge(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_plane(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
void launch_volume_top(const VolArgs &a, int idir, int jdir, int kdir, int mode, cudaStream_t st);
int launch_fault_pre(const FaultArgs &a, cudaStream_t st);
int launch_fault_post(const FaultArgs &a, cudaStream_t st);
cudaError_t noalloc_scratch_address(real **p);
void launch_record(const StationArgs &a, cudaStream_t st);
void launch_advance(Ctl *c, int max_rec, cudaStream_t st);
void launch_fault_gather(const real *out, real *dst, int nf, const Grid &g, cudaStream_t st);
int launch_sponge(const SpongeArgs &a, cudaStream_t st);
int launch_surface_peaks(const PeakArgs &a, cudaStream_t st);
}  // namespace cgfd

using namespace cgfd;

namespace {

thread_local std::string g_err;
// messages of cgfd_run_noalloc go to a fixed buffer (no allocation)
thread_local char g_err_fixed[256];
thread_local bool g_err_is_fixed = false;
int fail(int code, const std::string &m) { g_err = m; g_err_is_fixed = false; return code; }

// FD_Flags (src/forward/fd_t.cu:146-159): 0 backward, 1 forward
const int kPairs[8][3] = { {0,0,0},{1,1,0},{1,1,1},{0,0,1},{0,1,0},{1,0,0},{1,0,1},{0,1,1} };
const real kRkA[3] = { RL(0.5), RL(0.5), RL(1.0) };
const real kRkB[4] = { RL(1.0) / RL(6.0), RL(1.0) / RL(3.0), RL(1.0) / RL(3.0), RL(1.0) / RL(6.0) };

struct FaultState {
  FaultDev d;
  int j0 = 0, k0 = 0, nj = 0, nk = 0;   // bounding box of split nodes (interior)
  real *lev[4] = {};                    // storage slots, [9][2][ny*nz]
  uint8_t *flag = nullptr;
  real *mat = nullptr, *fmat = nullptr, *scal = nullptr, *out = nullptr;
  real *trac = nullptr;                 // traction scratch of the split box
  real *gather = nullptr;               // output fields at interior nodes, [11][nk][nj]
};

struct PmlState {
  PmlFaceDev d{};
  real *coef = nullptr;                 // A | B | D
  real *aux[4] = {};
};

}  // namespace

struct cgfd_solver {
  Grid g{};
  int imethod = 2, isfree = 0;
  float dt = 0.f, dtmax = 0.f;
  real *w[4] = {};                      // storage slots of the 4 levels
  real *coef = nullptr, *free_mat = nullptr;    // packed metric and medium (13 scmp values)
  real *abl_E = nullptr;                // sponge masks [nx | ny | nz]
  SpongeArgs sponge{};                  // sponge blocks (w set per step)
  real *pg = nullptr, *dis = nullptr;   // surface peaks [15][nj][ni], displacement [3][nj][ni]
  PmlState pml[6];
  std::vector<FaultState> faults;
  StationDev st{};
  long *sta_idx = nullptr;
  real *sta_w = nullptr, *fsta_w = nullptr;
  int *fsta_fid = nullptr, *fsta_idx = nullptr;
  real *seis = nullptr, *fseis = nullptr;
  Ctl *ctl = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph[2][8] = {};     // [timing][it % 8]
  bool use_graph = true;
  int timing = 0;
  cudaEvent_t ev_run[2] = {};
  cudaEvent_t ev_vol[8][4][2] = {};
  cudaEvent_t ev_int[8][4] = {};        // after the interior-box kernel
  cudaEvent_t ev_int0[8][4] = {};       // before it
  // concurrent branches of a stage: 0 none; 1 fault slabs and nodes, PML
  // slabs and shell beside the interior kernel; 2 the interior kernel
  // alone, then the fault slabs and nodes beside the PML slabs and shell;
  // 3 as 2 with the y and z PML slabs on a third stream from the interior
  // kernel's issue on (CGFD_BRANCHES): streams and fork / join events
  int branches = 3;
  cudaStream_t aux[3] = {};
  cudaEvent_t ev_fork[4] = {}, ev_join[4][3] = {}, ev_pre[4] = {};
  // the next stage's first fault kernels may overlap this stage's PML slab
  // and edge kernels (no fault neighbourhood meets their boxes)
  bool pre_early = false;
  // the interior kernel defers the fault planes x = i0 to a PLANE launch
  // and so runs beside the stage's first fault kernels (CGFD_PRE_OVERLAP)
  bool pre_overlap = false;
  // with pre_overlap: the fault slab kernels follow the stage's first fault
  // kernels on the fault stream at once, beside the interior kernel (and,
  // for stages 2-4, the previous stage's PML kernels), instead of after the
  // interior kernel (CGFD_POST_EARLY)
  bool post_early = true;
  cudaEvent_t ev_stage[4] = {}, ev_predone[4] = {}, ev_postdone[4] = {};
  double run_ms = 0, vol_ms = 0, int_ms = 0;
  long long vol_launches = 0, int_launches = 0;
  long long int_points = 0, vol_points = 0;   // points one launch updates
  int it = 0;
  long long launches_per_step = 0, last_launches = 0;
  int ychunk = 16;                      // interior kernel: y tiles per z-marching chunk (set at upload)
  bool pack = true;                     // pack boxes at most 24 points wide (x PML slabs)
  // boxes of each volume kernel kind: 0 interior, 1 generic shell (PML
  // edges / corners, surface rows), 2..4 slabs reached by the PML faces of
  // one direction only (x, y, z)
  int kbox[8][16][6];
  int nkbox[8] = {};
  std::vector<void *> allocs;
  // cgfd_run_fault_output: two device staging buffers of one record (all
  // faults' 11 fields at interior nodes), a copy stream and the events that
  // order gather -> copy -> reuse (made on first use)
  real *rec_buf[2] = {};
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_gathered[2] = {}, ev_copied[2] = {};
};

struct cgfd_setup {
  cgfd::HostSetup H;
  // the packed metric and medium (H.coef) moved to page-locked memory when
  // a device is present, so that cgfd_upload copies it at full link rate
  float *coef_pinned = nullptr;
  size_t coef_n = 0;
  const float *coef() const { return coef_pinned ? coef_pinned : H.coef.data(); }
  size_t coef_size() const { return coef_pinned ? coef_n : H.coef.size(); }
  ~cgfd_setup() { if (coef_pinned) cudaFreeHost(coef_pinned); }
};

namespace {

// host floats (the set-up's arrays) to device values of type real on the
// solver's stream; the double build widens them on the host first and
// copies synchronously
cudaError_t to_device(real *dst, const float *src, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
#ifdef CGFD_FP64
  std::vector<double> wide(src, src + n);
  cudaError_t e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? cudaMemcpy(dst, wide.data(), n * sizeof(double), cudaMemcpyHostToDevice) : e;
#else
  return cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyHostToDevice, st);
#endif
}

// device values of type real to host floats, waiting for the copy
cudaError_t to_host(float *dst, const real *src, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
#ifdef CGFD_FP64
  std::vector<double> wide(n);
  cudaError_t e = cudaMemcpyAsync(wide.data(), src, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) for (size_t q = 0; q < n; q++) dst[q] = (float)wide[q];
  return e;
#else
  cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost, st);
  return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
#endif
}

// Solver memory comes from the device's stream-ordered pool, which keeps
// freed blocks (release threshold at its maximum) so that a solver created
// after another one was destroyed reuses its memory instead of mapping new
// pages; cgfd_release_cached_memory hands the cached blocks back.
cudaError_t keep_pool_memory() {
  static std::atomic<unsigned long long> done{ 0 };
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev >= 64 || (done.load() & (1ull << dev))) return e;
  cudaMemPool_t pool;
  if ((e = cudaDeviceGetDefaultMemPool(&pool, dev)) != cudaSuccess) return e;
  unsigned long long thr = ~0ull;
  if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr)) != cudaSuccess) return e;
  done.fetch_or(1ull << dev);
  return cudaSuccess;
}

template <class T>
cudaError_t dalloc(cgfd_solver *s, T **p, size_t n) {
  cudaError_t e = keep_pool_memory();
  if (e == cudaSuccess) e = cudaMallocAsync((void **)p, std::max<size_t>(n, 1) * sizeof(T), s->stream);
  if (e == cudaSuccess) { s->allocs.push_back(*p); e = cudaMemsetAsync(*p, 0, std::max<size_t>(n, 1) * sizeof(T), s->stream); }
  return e;
}

// storage slot of logical level L (0 P, 1 A, 2 B, 3 E) at step parity
int slot(int L, int it) {
  if (L == LA || L == LB) return L;
  const bool odd = (it & 1) != 0;
  return (L == LP) != odd ? 0 : 3;
}

void destroy(cgfd_solver *s) {
  if (!s) return;
  for (int t = 0; t < 2; t++) for (int q = 0; q < 8; q++) if (s->graph[t][q]) cudaGraphExecDestroy(s->graph[t][q]);
  for (int q = 0; q < 2; q++) if (s->ev_run[q]) cudaEventDestroy(s->ev_run[q]);
  for (int a = 0; a < 8; a++) for (int b = 0; b < 4; b++) for (int c = 0; c < 2; c++)
    if (s->ev_vol[a][b][c]) cudaEventDestroy(s->ev_vol[a][b][c]);
  for (int a = 0; a < 8; a++) for (int b = 0; b < 4; b++) {
    if (s->ev_int[a][b]) cudaEventDestroy(s->ev_int[a][b]);
    if (s->ev_int0[a][b]) cudaEventDestroy(s->ev_int0[a][b]);
  }
  for (int a = 0; a < 4; a++) {
    if (s->ev_stage[a]) cudaEventDestroy(s->ev_stage[a]);
    if (s->ev_predone[a]) cudaEventDestroy(s->ev_predone[a]);
    if (s->ev_postdone[a]) cudaEventDestroy(s->ev_postdone[a]);
    if (s->ev_fork[a]) cudaEventDestroy(s->ev_fork[a]);
    if (s->ev_pre[a]) cudaEventDestroy(s->ev_pre[a]);
    for (int b = 0; b < 3; b++) if (s->ev_join[a][b]) cudaEventDestroy(s->ev_join[a][b]);
  }
  for (int q = 0; q < 3; q++) if (s->aux[q]) cudaStreamDestroy(s->aux[q]);
  for (int q = 0; q < 2; q++) {
    if (s->ev_gathered[q]) cudaEventDestroy(s->ev_gathered[q]);
    if (s->ev_copied[q]) cudaEventDestroy(s->ev_copied[q]);
  }
  if (s->copy) { cudaStreamSynchronize(s->copy); cudaStreamDestroy(s->copy); }
  for (void *p : s->allocs) cudaFreeAsync(p, s->stream);
  if (s->stream) {
    cudaStreamSynchronize(s->stream);
    cudaStreamDestroy(s->stream);
  }
  delete s;
}

// floats of traction scratch a fault's split box needs (12 planes x 9
// components over the box grown by 3 nodes); 0 for a fault without split
// nodes
size_t trac_floats(const FaultState &F) {
  return F.nj > 0 && F.nk > 0 ? (size_t)12 * 9 * (F.nj + 6) * (F.nk + 6) : 0;
}

// start of each fault's slice of a shared traction scratch: the slices lie
// one after another, each on a 64-float (256-byte) boundary; returns the
// floats all slices take
size_t trac_slices(const cgfd_solver *s, size_t *off) {
  size_t n = 0;
  for (size_t f = 0; f < s->faults.size(); f++) {
    off[f] = n;
    n += (trac_floats(s->faults[f]) + 63) / 64 * 64;
  }
  return n;
}

// enqueue one time step (graph capture or direct launches); trac: one
// traction scratch to use instead of each fault's own (cgfd_run_noalloc),
// split into one slice per fault because the first fault kernels of every
// fault run before the later ones of any fault; timed: whether the
// solver's timing events may be recorded
// the fault planes of a volume launch: x = i0 of each fault, its split-node
// flags and the deferred box (the split box grown by 3 nodes, empty when the
// fault has no split node)
void fault_planes(const cgfd_solver *s, VolArgs &v) {
  for (size_t f = 0; f < s->faults.size(); f++) {
    const FaultState &F = s->faults[f];
    v.fi0[f] = F.d.i0;
    v.fflag[f] = F.flag;
    const bool any = F.nj > 0 && F.nk > 0;
    v.fdef[f][0] = any ? F.j0 - 3 + NG : 1;
    v.fdef[f][1] = any ? F.j0 + F.nj + 2 + NG : 0;
    v.fdef[f][2] = any ? F.k0 - 3 + NG : 1;
    v.fdef[f][3] = any ? F.k0 + F.nk + 2 + NG : 0;
  }
}

void enqueue_step(cgfd_solver *s, int it, real *trac = nullptr, bool timed = true) {
  const int ip = it % 8;
  const bool tm = s->timing && timed;
  long long nl = 0;
  StationArgs sa{};
  sa.g = s->g; sa.st = s->st; sa.w = s->w[slot(LP, it)]; sa.ns = (long)s->g.ny * s->g.nz; sa.ctl = s->ctl;
  for (size_t f = 0; f < s->faults.size(); f++) sa.fout[f] = s->faults[f].out;
  if ((s->st.n + s->st.nf) > 0 && s->st.max_rec > 0) { launch_record(sa, s->stream); nl++; }
  // the fault kernels' arguments of one stage
  auto stage_fargs = [&](int stage, FaultArgs *fa) {
    const int idir = (kPairs[ip][0] + stage) % 2, jdir = (kPairs[ip][1] + stage) % 2, kdir = (kPairs[ip][2] + stage) % 2;
    const int mode = stage == 0 ? RK_FIRST : (stage == 3 ? RK_LAST : RK_MID);
    const int Lcur = stage == 0 ? LP : (stage == 2 ? LB : LA);
    const int Lout = stage == 0 ? LA : (stage == 1 ? LB : (stage == 2 ? LA : -1));
    const real ca = stage < 3 ? kRkA[stage] * s->dt : RL(0.0), cb = kRkB[stage] * s->dt;
    const int scur = slot(Lcur, it), spre = slot(LP, it), send = slot(LE, it);
    const int sout = Lout >= 0 ? slot(Lout, it) : -1;
    size_t toff[MAXF] = {};
    if (trac) trac_slices(s, toff);
    int n = 0;
    for (auto &F : s->faults) {
      const size_t myoff = toff[n];
      FaultArgs &a = fa[n++];
      a = FaultArgs{};
      a.g = s->g; a.F = F.d;
      a.wcur = s->w[scur]; a.wpre = s->w[spre]; a.wout = sout >= 0 ? s->w[sout] : nullptr; a.wend = s->w[send];
      a.coef = s->coef; a.free_mat = s->free_mat;
      a.fc = F.lev[scur]; a.fp = F.lev[spre]; a.fo = sout >= 0 ? F.lev[sout] : nullptr; a.fe = F.lev[send];
      a.idir = idir; a.jdir = jdir; a.kdir = kdir; a.mode = mode;
      a.ca = ca; a.cb = cb; a.rkb = kRkB[stage]; a.dt = s->dt;
      a.isfree = s->isfree; a.imethod = s->imethod;
      a.j0 = F.j0; a.k0 = F.k0; a.nj = F.nj; a.nk = F.nk; a.ctl = s->ctl;
      a.trac = trac ? trac + myoff : F.trac; a.tj0 = F.j0 + NG - 3; a.tk0 = F.k0 + NG - 3; a.tnj = F.nj + 6; a.tnk = F.nk + 6;
      if (F.nj > 0 && F.nk > 0) {
        a.wj0 = std::max(0, F.j0 - 3); a.wk0 = std::max(0, F.k0 - 3);
        a.wnj = std::min(s->g.nj - 1, F.j0 + F.nj + 2) - a.wj0 + 1;
        a.wnk = std::min(s->g.nk - 1, F.k0 + F.nk + 2) - a.wk0 + 1;
      } else {
        a.wj0 = 0; a.wk0 = 0; a.wnj = s->g.nj; a.wnk = s->g.nk;
      }
    }
    return n;
  };
  // branches: after the trial traction (which refreshes the stage input
  // at the split nodes), the fault slabs and nodes, the interior kernel
  // and the PML slabs / shell read the same input and write disjoint
  // points, so they may run on separate streams joined before the next
  // stage.  With pre_early, the next stage's first fault kernels (which
  // read only the fault's neighbourhood, away from every PML slab and
  // edge box) start on the fault stream once this stage's interior,
  // surface-row and fault kernels are done, beside its PML and edge kernels.
  // branches 3: as 2, and the y and z PML slab kernels run on a third
  // stream beside the x slab, edge and surface-row kernels (disjoint
  // points, the same input), so that their launch gaps and tails overlap
  // (the default).  With post_early the fault slab kernels follow the first
  // fault kernels on the fault stream at once: the slab points' input is
  // complete then, and the lines of the fault neighbourhood that the first
  // kernels brought into L2 are still there
  const bool br = s->branches == 1, br2 = s->branches >= 2, br3 = s->branches == 3;
  const bool early = br2 && s->pre_early;
  const bool ov = br2 && s->pre_overlap;
  const bool pe2 = ov && s->post_early;
  FaultArgs fargs[MAXF], fnext[MAXF];
  const int nfa = stage_fargs(0, fargs);
  for (int stage = 0; stage < 4; stage++) {
    const int idir = (kPairs[ip][0] + stage) % 2, jdir = (kPairs[ip][1] + stage) % 2, kdir = (kPairs[ip][2] + stage) % 2;
    const int mode = stage == 0 ? RK_FIRST : (stage == 3 ? RK_LAST : RK_MID);
    const int Lcur = stage == 0 ? LP : (stage == 2 ? LB : LA);
    const int Lout = stage == 0 ? LA : (stage == 1 ? LB : (stage == 2 ? LA : -1));
    const real ca = stage < 3 ? kRkA[stage] * s->dt : RL(0.0), cb = kRkB[stage] * s->dt;
    const int scur = slot(Lcur, it), spre = slot(LP, it), send = slot(LE, it);
    const int sout = Lout >= 0 ? slot(Lout, it) : -1;
    if (stage > 0) {
      if (early) std::memcpy(fargs, fnext, sizeof(FaultArgs) * nfa);
      else stage_fargs(stage, fargs);
    }
    if (!(early && stage > 0)) {
      if (ov) {
        // on the fault stream, beside the interior kernel (which defers the
        // fault planes), once the stage input is complete
        cudaEventRecord(s->ev_stage[stage], s->stream);
        cudaStreamWaitEvent(s->aux[0], s->ev_stage[stage], 0);
        for (int f = 0; f < nfa; f++) nl += launch_fault_pre(fargs[f], s->aux[0]);
        cudaEventRecord(s->ev_predone[stage], s->aux[0]);
        if (pe2) {
          for (int f = 0; f < nfa; f++) nl += launch_fault_post(fargs[f], s->aux[0]);
          cudaEventRecord(s->ev_postdone[stage], s->aux[0]);
        }
      } else {
        for (int f = 0; f < nfa; f++) nl += launch_fault_pre(fargs[f], s->stream);
      }
    }
    // external event nodes when captured, so that the events really fire
    // on every graph replay; the stage interval spans the fork to the join
    if (tm) cudaEventRecordWithFlags(s->ev_vol[ip][stage][0], s->stream, cudaEventRecordExternal);
    cudaStream_t st_int = s->stream, st_fault = s->stream, st_pml = s->stream;
    if (br) {
      st_fault = s->aux[0];
      st_pml = s->aux[1];
      cudaEventRecord(s->ev_fork[stage], s->stream);
      cudaStreamWaitEvent(st_fault, s->ev_fork[stage], 0);
      cudaStreamWaitEvent(st_pml, s->ev_fork[stage], 0);
    }
    if (!br2)
      for (int f = 0; f < nfa; f++) nl += launch_fault_post(fargs[f], st_fault);
    VolArgs v{};
    v.g = s->g; v.cur = s->w[scur]; v.pre = s->w[spre]; v.out = sout >= 0 ? s->w[sout] : nullptr; v.end = s->w[send];
    v.coef = s->coef; v.free_mat = s->free_mat;
    v.ca = ca; v.cb = cb; v.isfree = s->isfree;
    v.nfault = (int)s->faults.size();
    v.defer_i0 = ov ? 1 : 0;
    fault_planes(s, v);
    for (int q = 0; q < 6; q++) {
      v.pml[q] = s->pml[q].d;
      if (!v.pml[q].on) continue;
      v.pml[q].acur = s->pml[q].aux[scur]; v.pml[q].apre = s->pml[q].aux[spre];
      v.pml[q].aout = sout >= 0 ? s->pml[q].aux[sout] : nullptr; v.pml[q].aend = s->pml[q].aux[send];
    }
    VolArgs vs = v;
    {
      // interior box, single-direction PML slabs, generic shell
      const int kind0 = 0;
      for (int kind = kind0; kind < 6; kind++) {
        if (kind == 1 && ov) {
          // the fault planes x = i0 once the stage's first fault kernels
          // (which refresh the split nodes there) are done
          cudaStreamWaitEvent(s->stream, s->ev_predone[stage], 0);
          VolArgs vp = vs;
          volume_boxes(vp, s->kbox[6], s->nkbox[6], true);
          if (vp.nbox > 0) { launch_volume_plane(vp, idir, jdir, kdir, mode, s->stream); nl++; }
        }
        if (kind == 1 && br2) {
          // the interior kernel has been issued alone; the fault kernels
          // now overlap the PML slabs and the shell
          st_fault = s->aux[0];
          cudaEventRecord(s->ev_fork[stage], s->stream);
          if (br3) cudaStreamWaitEvent(s->aux[1], s->ev_fork[stage], 0);
          if (!pe2) {
            cudaStreamWaitEvent(st_fault, s->ev_fork[stage], 0);
            for (int f = 0; f < nfa; f++) nl += launch_fault_post(fargs[f], st_fault);
            if (ov) cudaEventRecord(s->ev_postdone[stage], st_fault);
          }
        }
        if (kind == 2 && early && stage < 3) {
          // the surface rows are issued: the next stage's input is complete
          // in the fault's neighbourhood once they and the fault kernels end
          cudaEventRecord(s->ev_pre[stage], s->stream);
          cudaStreamWaitEvent(st_fault, s->ev_pre[stage], 0);
          stage_fargs(stage + 1, fnext);
          for (int f = 0; f < nfa; f++) nl += launch_fault_pre(fnext[f], st_fault);
          if (ov) cudaEventRecord(s->ev_predone[stage + 1], st_fault);
          if (pe2) {
            // the slab points' input is complete as well (the PML boxes
            // and their stencils stay clear of the fault neighbourhood), and
            // no kernel of this stage reads or writes the next stage's
            // output or end level there
            for (int f = 0; f < nfa; f++) nl += launch_fault_post(fnext[f], st_fault);
            cudaEventRecord(s->ev_postdone[stage + 1], st_fault);
          }
        }
        if (kind == 1) {
          // surface rows away from every PML face, beside (before) the
          // shell's rows in the PML columns
          VolArgs vt = vs;
          volume_boxes(vt, s->kbox[7], s->nkbox[7], s->pack);
          if (vt.nbox > 0) { launch_volume_top(vt, idir, jdir, kdir, mode, st_pml); nl++; }
        }
        VolArgs vk = vs;
        volume_boxes(vk, s->kbox[kind], s->nkbox[kind], kind != 0 && s->pack);
        vk.ychunk = s->ychunk;
        if (vk.nbox == 0) continue;
        switch (kind) {
          case 0:
            if (tm) cudaEventRecordWithFlags(s->ev_int0[ip][stage], st_int, cudaEventRecordExternal);
            launch_volume_interior(vk, idir, jdir, kdir, mode, st_int);
            if (tm) cudaEventRecordWithFlags(s->ev_int[ip][stage], st_int, cudaEventRecordExternal);
            break;
          case 1: launch_volume_shell(vk, idir, jdir, kdir, mode, st_pml); break;
          case 2: launch_volume_face_x(vk, idir, jdir, kdir, mode, st_pml); break;
          case 3: launch_volume_face_y(vk, idir, jdir, kdir, mode, br3 ? s->aux[1] : st_pml); break;
          case 4: launch_volume_face_z(vk, idir, jdir, kdir, mode, br3 ? s->aux[1] : st_pml); break;
          default: launch_volume_edge(vk, idir, jdir, kdir, mode, st_pml); break;
        }
        nl += vk.nbox > 0;
      }
    }
    if (br) {
      cudaEventRecord(s->ev_join[stage][0], st_fault);
      cudaEventRecord(s->ev_join[stage][1], st_pml);
      cudaStreamWaitEvent(s->stream, s->ev_join[stage][0], 0);
      cudaStreamWaitEvent(s->stream, s->ev_join[stage][1], 0);
    } else if (br2) {
      // with the fault planes deferred, the stage ends when the fault slab
      // kernels end: the next stage's early first fault kernels, queued
      // behind them, only have to end before its PLANE launch
      if (ov) {
        cudaStreamWaitEvent(s->stream, s->ev_postdone[stage], 0);
      } else {
        cudaEventRecord(s->ev_join[stage][0], st_fault);
        cudaStreamWaitEvent(s->stream, s->ev_join[stage][0], 0);
      }
      if (br3) {
        cudaEventRecord(s->ev_join[stage][1], s->aux[1]);
        cudaStreamWaitEvent(s->stream, s->ev_join[stage][1], 0);
      }
    }
    if (tm) cudaEventRecordWithFlags(s->ev_vol[ip][stage][1], s->stream, cudaEventRecordExternal);
  }
  // end of step on the time n+1 level: sponge, then the surface peaks
  // (drv_rk_curv_col.cu:600-613)
  if (s->sponge.nblk > 0) {
    SpongeArgs sp = s->sponge;
    sp.w = s->w[slot(LE, it)];
    nl += launch_sponge(sp, s->stream);
  }
  if (s->isfree) {
    PeakArgs pa{};
    pa.g = s->g; pa.wend = s->w[slot(LE, it)]; pa.wpre = s->w[slot(LP, it)];
    pa.pg = s->pg; pa.dis = s->dis; pa.dt = s->dt;
    nl += launch_surface_peaks(pa, s->stream);
  }
  launch_advance(s->ctl, s->st.max_rec, s->stream);
  nl++;
  s->launches_per_step = nl;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int cgfd_abi_version(void) { return CGFD_ABI_VERSION; }

void cgfd_config_default(cgfd_config *c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->check_stability = 1;
  c->dynamic_method = 2;
  c->welded_margin = 40;
  c->grid_mode = CGFD_GRID_FAULT_PLANE;
  for (int d = 0; d < 3; d++) for (int s = 0; s < 2; s++) {
    c->pml_alpha_max[d][s] = 3.14f; c->pml_beta_max[d][s] = 2.0f; c->pml_ref_vel[d][s] = 6000.f;
    c->ablexp_ref_vel[d][s] = 6000.f;
  }
}

const char *cgfd_last_error(void) { return g_err_is_fixed ? g_err_fixed : g_err.c_str(); }

int cgfd_prepare(const cgfd_config *cfg, cgfd_setup **out) {
  if (!cfg || !out) return fail(CGFD_ERR_ARG, "null argument");
  *out = nullptr;
  cgfd_setup *su = new cgfd_setup();
  std::string msg;
  int rc = build_setup(cfg, su->H, msg);
  if (rc != CGFD_OK) { delete su; return fail(rc, msg); }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
    float *pc = nullptr;
    const size_t n = su->H.coef.size();
    if (cudaMallocHost((void **)&pc, n * sizeof(float)) == cudaSuccess) {
      std::memcpy(pc, su->H.coef.data(), n * sizeof(float));
      su->coef_pinned = pc;
      su->coef_n = n;
      std::vector<float>().swap(su->H.coef);
    }
  }
  cudaGetLastError();   // no device, or no page-locked memory: keep the vector
  *out = su;
  return CGFD_OK;
}

void cgfd_setup_free(cgfd_setup *su) { delete su; }

int cgfd_setup_dt_max(const cgfd_setup *su, float *d) {
  if (!su || !d) return fail(CGFD_ERR_ARG, "bad argument");
  *d = su->H.dtmax;
  return CGFD_OK;
}

int cgfd_release_cached_memory(void) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  cudaMemPool_t pool;
  if (e == cudaSuccess) e = cudaDeviceGetDefaultMemPool(&pool, dev);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
  return e == cudaSuccess ? CGFD_OK : cuda_fail(e, "release cached memory");
}

int cgfd_select_device(int ordinal) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(CGFD_ERR_NODEVICE, "no CUDA device");
  if (ordinal < 0 || ordinal >= n) return fail(CGFD_ERR_ARG, "device ordinal out of range");
  e = cudaSetDevice(ordinal);
  if (e != cudaSuccess) return cuda_fail(e, "select device");
  return CGFD_OK;
}

int cgfd_setup_coords(const cgfd_setup *su, float *x, float *y, float *z) {
  if (!su) return fail(CGFD_ERR_ARG, "bad argument");
  const size_t np = su->H.coords.size() / 3;
  if (x) std::memcpy(x, su->H.coords.data(), np * 4);
  if (y) std::memcpy(y, su->H.coords.data() + np, np * 4);
  if (z) std::memcpy(z, su->H.coords.data() + 2 * np, np * 4);
  return CGFD_OK;
}

int cgfd_setup_bytes(const cgfd_setup *su, unsigned long long *bytes) {
  if (!su || !bytes) return fail(CGFD_ERR_ARG, "bad argument");
  const HostSetup &H = su->H;
  const unsigned long long R = sizeof(real);
  unsigned long long n = (su->coef_size() + H.free_mat.size()) * R;
  for (int d = 0; d < 3; d++) for (int q = 0; q < 2; q++) n += 3ull * (H.pml[d][q].A.size()) * R;
  for (auto &F : H.faults) n += F.flag.size() + (F.mat.size() + F.fmat.size() + F.scal.size() + F.out.size()) * R;
  n += H.sta_idx.size() * sizeof(long) + (H.sta_w.size() + H.fsta_w.size()) * R + (H.fsta_fid.size() + H.fsta_idx.size()) * 4ull;
  *bytes = n;
  return CGFD_OK;
}

int cgfd_create(const cgfd_config *cfg, cgfd_solver **out) {
  if (!cfg || !out) return fail(CGFD_ERR_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(CGFD_ERR_NODEVICE, "no CUDA device visible");
  }
  cgfd_setup *su = nullptr;
  int rc = cgfd_prepare(cfg, &su);
  if (rc != CGFD_OK) return rc;
  rc = cgfd_upload(su, out);
  cgfd_setup_free(su);
  return rc;
}

static int build_graphs(cgfd_solver *s);


// Autotuner of the interior kernel's y chunk (the number of 8-row tiles whose
// blocks march up z together, which sets how much of L2 the stencil planes
// take): the first stage's interior launch is timed for a few chunk sizes
// on the solver's state at upload, which is all zero, so the launches write
// zeros where zeros are and change nothing.  The fastest size is kept per
// device and interior box, so later solvers of the same shape reuse it.
static std::mutex g_tune_mu;
static std::map<std::array<int, 4>, int> g_tune;

static cudaError_t tune_ychunk(cgfd_solver *s) {
  if (s->nkbox[0] == 0) return cudaSuccess;
  const int *B = s->kbox[0][0];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const std::array<int, 4> key = { dev, B[1] - B[0] + 1, B[3] - B[2] + 1, B[5] - B[4] + 1 };
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto f = g_tune.find(key);
    if (f != g_tune.end()) { s->ychunk = f->second; return cudaSuccess; }
  }
  const int ntiles = (key[2] + 7) / 8, ip = s->it % 8, it = s->it;
  VolArgs v{};
  v.g = s->g; v.cur = s->w[slot(LP, it)]; v.pre = v.cur; v.out = s->w[slot(LA, it)]; v.end = s->w[slot(LE, it)];
  v.coef = s->coef; v.free_mat = s->free_mat;
  v.ca = kRkA[0] * s->dt; v.cb = kRkB[0] * s->dt; v.isfree = s->isfree;
  v.nfault = (int)s->faults.size();
  fault_planes(s, v);
  volume_boxes(v, s->kbox[0], s->nkbox[0], false);
  cudaEvent_t t0, t1;
  if ((e = cudaEventCreate(&t0)) != cudaSuccess) return e;
  if ((e = cudaEventCreate(&t1)) != cudaSuccess) { cudaEventDestroy(t0); return e; }
  int best = s->ychunk;
  float best_ms = 1e30f;
  std::vector<int> cand;
  for (int c : { 8, 16, 32, 64, ntiles }) {
    c = std::max(1, std::min(c, ntiles));
    if (std::find(cand.begin(), cand.end(), c) == cand.end()) cand.push_back(c);
  }
  for (int c : cand) {
    v.ychunk = c;
    launch_volume_interior(v, kPairs[ip][0], kPairs[ip][1], kPairs[ip][2], RK_FIRST, s->stream);
    cudaEventRecord(t0, s->stream);
    for (int r = 0; r < 2; r++) launch_volume_interior(v, kPairs[ip][0], kPairs[ip][1], kPairs[ip][2], RK_FIRST, s->stream);
    cudaEventRecord(t1, s->stream);
    if ((e = cudaEventSynchronize(t1)) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    if (ms < best_ms) { best_ms = ms; best = c; }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  s->ychunk = best;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  return cudaSuccess;
}

int cgfd_upload(const cgfd_setup *su, cgfd_solver **out) {
  if (!su || !out) return fail(CGFD_ERR_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(CGFD_ERR_NODEVICE, "no CUDA device visible");
  }
  const HostSetup &H = su->H;
  cgfd_solver *s = new cgfd_solver();
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { destroy(s); return cuda_fail(e, "stream"); }
  s->g = H.g; s->imethod = H.imethod; s->isfree = H.isfree; s->dt = H.dt; s->dtmax = H.dtmax;
  const char *ng = std::getenv("CGFD_NO_GRAPH");
  s->use_graph = !(ng && ng[0] == '1');
  const Grid &g = s->g;
  const size_t lev = (size_t)NCMP * g.scmp, ns = (size_t)g.ny * g.nz;
#define CK(x, what) do { cudaError_t _e = (x); if (_e != cudaSuccess) { destroy(s); return cuda_fail(_e, what); } } while (0)
  for (int L = 0; L < 4; L++) CK(dalloc(s, &s->w[L], lev), "wavefield");
  CK(dalloc(s, &s->coef, 13 * (size_t)g.scmp), "metric");
  CK(dalloc(s, &s->free_mat, H.free_mat.size()), "free surface");
  CK(to_device(s->coef, su->coef(), su->coef_size(), s->stream), "copy metric");
  CK(to_device(s->free_mat, H.free_mat.data(), H.free_mat.size(), s->stream), "copy free");
  if (H.abl_nblk > 0) {
    CK(dalloc(s, &s->abl_E, (size_t)g.nx + g.ny + g.nz), "sponge");
    CK(to_device(s->abl_E, H.abl_E[0].data(), g.nx, s->stream), "copy sponge");
    CK(to_device(s->abl_E + g.nx, H.abl_E[1].data(), g.ny, s->stream), "copy sponge");
    CK(to_device(s->abl_E + g.nx + g.ny, H.abl_E[2].data(), g.nz, s->stream), "copy sponge");
    SpongeArgs &sp = s->sponge;
    sp.g = g; sp.E = s->abl_E; sp.nblk = H.abl_nblk;
    sp.first[0] = 0;
    for (int b = 0; b < H.abl_nblk; b++) {
      const int *B = H.abl_blk[b];
      for (int q = 0; q < 6; q++) sp.blk[b][q] = B[q];
      sp.first[b + 1] = sp.first[b] + (long)(B[1] - B[0] + 1) * (B[3] - B[2] + 1) * (B[5] - B[4] + 1);
    }
  }
  if (H.isfree) {
    CK(dalloc(s, &s->pg, (size_t)CGFD_NPEAK * g.ni * g.nj), "surface peaks");
    CK(dalloc(s, &s->dis, (size_t)3 * g.ni * g.nj), "surface displacement");
  }
  for (int d = 0; d < 3; d++) for (int sd = 0; sd < 2; sd++) {
    const PmlHost &P = H.pml[d][sd];
    PmlState &S = s->pml[2 * d + sd];
    S.d.on = P.on; S.d.d = d; S.d.s = sd; S.d.L = P.L;
    if (!P.on) continue;
    S.d.i1 = P.i1; S.d.j1 = P.j1; S.d.k1 = P.k1;
    S.d.fni = P.i2 - P.i1 + 1; S.d.fnj = P.j2 - P.j1 + 1; S.d.fnk = P.k2 - P.k1 + 1;
    S.d.siz = (long)S.d.fni * S.d.fnj * S.d.fnk;
    const int np = P.L + 1;
    CK(dalloc(s, &S.coef, 3 * (size_t)np), "pml coef");
    std::vector<float> cf(3 * np);
    std::copy(P.A.begin(), P.A.end(), cf.begin());
    std::copy(P.B.begin(), P.B.end(), cf.begin() + np);
    std::copy(P.D.begin(), P.D.end(), cf.begin() + 2 * np);
    CK(to_device(S.coef, cf.data(), cf.size(), s->stream), "copy pml");
    S.d.A = S.coef; S.d.B = S.coef + np; S.d.D = S.coef + 2 * np;
    for (int L = 0; L < 4; L++) CK(dalloc(s, &S.aux[L], (size_t)NCMP * S.d.siz), "pml aux");
  }
  for (size_t f = 0; f < H.faults.size(); f++) {
    const FaultHost &Fh = H.faults[f];
    FaultState F;
    for (int L = 0; L < 4; L++) CK(dalloc(s, &F.lev[L], 18 * ns), "fault wavefield");
    CK(dalloc(s, &F.flag, ns), "fault flags");
    CK(dalloc(s, &F.mat, Fh.mat.size()), "fault matrices");
    CK(dalloc(s, &F.fmat, Fh.fmat.size()), "fault free matrices");
    CK(dalloc(s, &F.scal, Fh.scal.size()), "fault scalars");
    CK(dalloc(s, &F.out, Fh.out.size()), "fault output");
    CK(cudaMemcpyAsync(F.flag, Fh.flag.data(), ns, cudaMemcpyHostToDevice, s->stream), "copy");
    CK(to_device(F.mat, Fh.mat.data(), Fh.mat.size(), s->stream), "copy");
    CK(to_device(F.fmat, Fh.fmat.data(), Fh.fmat.size(), s->stream), "copy");
    CK(to_device(F.scal, Fh.scal.data(), Fh.scal.size(), s->stream), "copy");
    CK(to_device(F.out, Fh.out.data(), Fh.out.size(), s->stream), "copy");
    F.d.i0 = Fh.i0; F.d.bit = 1 << f; F.d.flag_in = F.flag; F.d.flag = F.flag;
    F.d.mat = F.mat; F.d.fmat = F.fmat; F.d.scal = F.scal; F.d.out = F.out;
    int j0 = g.nj, j1 = -1, k0 = g.nk, k1 = -1;
    for (int k = 0; k < g.nk; k++) for (int j = 0; j < g.nj; j++)
      if (Fh.flag[(size_t)(j + NG) + (size_t)(k + NG) * g.ny] & FL_SPLIT) {
        j0 = std::min(j0, j); j1 = std::max(j1, j); k0 = std::min(k0, k); k1 = std::max(k1, k);
      }
    if (j1 >= 0) {
      F.j0 = j0; F.k0 = k0; F.nj = j1 - j0 + 1; F.nk = k1 - k0 + 1;
      CK(dalloc(s, &F.trac, (size_t)12 * 9 * (F.nj + 6) * (F.nk + 6)), "fault traction scratch");
    }
    CK(dalloc(s, &F.gather, (size_t)CGFD_FAULT_NFIELD * g.nj * g.nk), "fault output staging");
    s->faults.push_back(F);
  }
  // stations
  StationDev &st = s->st;
  st.n = (int)(H.sta_w.size() / 3); st.nf = (int)H.fsta_fid.size(); st.max_rec = H.max_rec;
  CK(dalloc(s, &s->sta_idx, H.sta_idx.size()), "stations");
  CK(dalloc(s, &s->sta_w, H.sta_w.size()), "stations");
  CK(dalloc(s, &s->fsta_fid, H.fsta_fid.size()), "stations");
  CK(dalloc(s, &s->fsta_idx, H.fsta_idx.size()), "stations");
  CK(dalloc(s, &s->fsta_w, H.fsta_w.size()), "stations");
  CK(dalloc(s, &s->seis, (size_t)st.n * 9 * std::max(1, st.max_rec)), "seismograms");
  CK(dalloc(s, &s->fseis, (size_t)st.nf * 9 * std::max(1, st.max_rec)), "fault seismograms");
  if (!H.sta_idx.empty()) {
    CK(cudaMemcpyAsync(s->sta_idx, H.sta_idx.data(), H.sta_idx.size() * sizeof(long), cudaMemcpyHostToDevice, s->stream), "copy");
    CK(to_device(s->sta_w, H.sta_w.data(), H.sta_w.size(), s->stream), "copy");
  }
  if (!H.fsta_fid.empty()) {
    CK(cudaMemcpyAsync(s->fsta_fid, H.fsta_fid.data(), H.fsta_fid.size() * 4, cudaMemcpyHostToDevice, s->stream), "copy");
    CK(cudaMemcpyAsync(s->fsta_idx, H.fsta_idx.data(), H.fsta_idx.size() * 4, cudaMemcpyHostToDevice, s->stream), "copy");
    CK(to_device(s->fsta_w, H.fsta_w.data(), H.fsta_w.size(), s->stream), "copy");
  }
  st.idx = s->sta_idx; st.w = s->sta_w; st.fid = s->fsta_fid; st.fidx = s->fsta_idx; st.fw = s->fsta_w;
  st.seis = s->seis; st.fseis = s->fseis;
  // boxes of the volume kernel kinds (interior indices, inclusive)
  {
    auto L = [&](int d, int sd) { return H.pml[d][sd].on ? H.pml[d][sd].L + 1 : 0; };
    const int ilo = L(0, 0), ihi = g.ni - 1 - L(0, 1), jlo = L(1, 0), jhi = g.nj - 1 - L(1, 1);
    const int klo = L(2, 0), khi = s->isfree ? g.nk - 5 : g.nk - 1 - L(2, 1);
    bool box_overflow = false;
    auto add = [&](int kind, int i0, int i1, int j0, int j1, int k0, int k1) {
      if (i1 < i0 || j1 < j0 || k1 < k0) return;
      if (s->nkbox[kind] >= 16) { box_overflow = true; return; }
      int *b = s->kbox[kind][s->nkbox[kind]++];
      b[0] = i0; b[1] = i1; b[2] = j0; b[3] = j1; b[4] = k0; b[5] = k1;
    };
    const int ni = g.ni, nj = g.nj, nk = g.nk;
    // the interior box is a whole number of 32-point tiles wide in x; the
    // columns left over (fewer than 32) join the right x PML slab, not a last
    // tile of each row whose warps would have only those few lanes at work
    // (unless a fault's neighbourhood reaches them: the fault kernels may
    // start beside the PML kernels only away from their boxes).  The y and z
    // PML slabs and the surface rows over the interior box's x extent are
    // cut the same way, their leftover columns going to the generic edge and
    // shell kernels
    int iha = ihi;
    {
      const int w = ihi - ilo + 1, wa = w / 32 * 32;
      const char *at = std::getenv("CGFD_ALIGN_TILES");
      bool split = wa > 0 && wa < w && !(at && at[0] == '0');
      for (auto &F : s->faults)
        if (F.d.i0 - NG + 6 >= ilo + wa && F.d.i0 - NG - 6 <= ihi) split = false;
      if (split) iha = ilo + wa - 1;
    }
    add(0, ilo, iha, jlo, jhi, klo, khi);
    // one PML direction only
    add(2, 0, ilo - 1, jlo, jhi, klo, khi);
    add(2, iha + 1, ni - 1, jlo, jhi, klo, khi);
    add(3, ilo, iha, 0, jlo - 1, klo, khi);
    add(3, ilo, iha, jhi + 1, nj - 1, klo, khi);
    add(4, ilo, iha, jlo, jhi, 0, klo - 1);
    if (!s->isfree) add(4, ilo, iha, jlo, jhi, khi + 1, nk - 1);
    add(5, iha + 1, ihi, 0, jlo - 1, klo, khi);
    add(5, iha + 1, ihi, jhi + 1, nj - 1, klo, khi);
    add(5, iha + 1, ihi, jlo, jhi, 0, klo - 1);
    if (!s->isfree) add(5, iha + 1, ihi, jlo, jhi, khi + 1, nk - 1);
    // vertical edges, bottom ring, top ring (edge kernel); surface rows
    // (shell kernel)
    add(5, 0, ilo - 1, 0, jlo - 1, klo, khi);
    add(5, 0, ilo - 1, jhi + 1, nj - 1, klo, khi);
    add(5, ihi + 1, ni - 1, 0, jlo - 1, klo, khi);
    add(5, ihi + 1, ni - 1, jhi + 1, nj - 1, klo, khi);
    add(5, 0, ilo - 1, 0, nj - 1, 0, klo - 1);
    add(5, ihi + 1, ni - 1, 0, nj - 1, 0, klo - 1);
    add(5, ilo, ihi, 0, jlo - 1, 0, klo - 1);
    add(5, ilo, ihi, jhi + 1, nj - 1, 0, klo - 1);
    const char *tp = std::getenv("CGFD_TOP");
    if (s->isfree && khi + 1 >= klo && !(tp && tp[0] == '0')) {
      // the rows of the PML columns (shell) and the rest (top kernel)
      add(7, ilo, iha, jlo, jhi, khi + 1, nk - 1);
      add(1, iha + 1, ihi, jlo, jhi, khi + 1, nk - 1);
      add(1, 0, ilo - 1, 0, nj - 1, khi + 1, nk - 1);
      add(1, ihi + 1, ni - 1, 0, nj - 1, khi + 1, nk - 1);
      add(1, ilo, ihi, 0, jlo - 1, khi + 1, nk - 1);
      add(1, ilo, ihi, jhi + 1, nj - 1, khi + 1, nk - 1);
    } else if (s->isfree) {
      add(1, 0, ni - 1, 0, nj - 1, khi + 1, nk - 1);
    } else {
      add(5, 0, ilo - 1, 0, nj - 1, khi + 1, nk - 1);
      add(5, ihi + 1, ni - 1, 0, nj - 1, khi + 1, nk - 1);
      add(5, ilo, ihi, 0, jlo - 1, khi + 1, nk - 1);
      add(5, ilo, ihi, jhi + 1, nj - 1, khi + 1, nk - 1);
    }
    if (box_overflow) { destroy(s); return fail(CGFD_ERR_ARG, "too many volume boxes of one kind"); }
    // a stage's first fault kernels read its input at i0-6..i0+6 over the
    // split box grown by 3 nodes: when that region meets no PML slab or edge
    // box for any fault, they may start before those kernels of the
    // previous stage end
    s->pre_early = !s->faults.empty();
    for (auto &F : s->faults) {
      if (F.nj <= 0 || F.nk <= 0) { s->pre_early = false; break; }
      const int r[6] = { F.d.i0 - NG - 6, F.d.i0 - NG + 6, F.j0 - 3, F.j0 + F.nj + 2, F.k0 - 3, F.k0 + F.nk + 2 };
      for (int kind = 2; kind < 6; kind++)
        for (int b = 0; b < s->nkbox[kind]; b++) {
          const int *B = s->kbox[kind][b];
          if (B[0] <= r[1] && r[0] <= B[1] && B[2] <= r[3] && r[2] <= B[3] && B[4] <= r[5] && r[4] <= B[5])
            s->pre_early = false;
        }
    }
    const char *pe = std::getenv("CGFD_PRE_EARLY");
    if (pe && pe[0] == '0') s->pre_early = false;
    // the fault planes inside the interior box within the split boxes grown
    // by 3 nodes, for the PLANE launch when the interior kernel defers them
    for (auto &F : s->faults) {
      const int ii = F.d.i0 - NG;
      if (ii >= ilo && ii <= iha && F.nj > 0 && F.nk > 0)
        add(6, ii, ii, std::max(jlo, F.j0 - 3), std::min(jhi, F.j0 + F.nj + 2), std::max(klo, F.k0 - 3),
            std::min(khi, F.k0 + F.nk + 2));
    }
    s->pre_overlap = !s->faults.empty();
    const char *po = std::getenv("CGFD_PRE_OVERLAP");
    if (po && po[0] == '0') s->pre_overlap = false;
    const char *pq = std::getenv("CGFD_POST_EARLY");
    if (pq && pq[0] == '0') s->post_early = false;
    const char *pk = std::getenv("CGFD_PACK");
    if (pk && pk[0] == '0') s->pack = false;
    // y tiles (8 rows) per interior chunk: the z window of a chunk, about 8
    // planes of the stage input (36 B a point), should take at most ~24 MB
    // of the 126 MB L2, which also carries the streamed arrays (measured:
    // 1200x600x400 best at 16-24 tiles, 600x300x240 at its whole plane)
    {
      const long row_bytes = (long)std::max(1, ihi - ilo + 1) * 8 * 36;
      s->ychunk = (int)std::max(4L, (24L << 20) / (8 * row_bytes));
    }
    const char *yc = std::getenv("CGFD_INTERIOR_YCHUNK");
    if (yc && std::atoi(yc) > 0) s->ychunk = std::atoi(yc);
    s->ychunk = std::min(s->ychunk, std::max(1, (jhi - jlo + 8) / 8));
    // points one interior launch / one volume stage updates: the split-node
    // slabs belong to the fault kernels
    long long nint = (long long)std::max(0, iha - ilo + 1) * std::max(0, jhi - jlo + 1) * std::max(0, khi - klo + 1);
    long long nall = (long long)ni * nj * nk;
    for (size_t f = 0; f < H.faults.size(); f++) {
      const FaultHost &Fh = H.faults[f];
      for (int k = 0; k < nk; k++) for (int j = 0; j < nj; j++) {
        if (!(Fh.flag[(size_t)(j + NG) + (size_t)(k + NG) * g.ny] & FL_SPLIT)) continue;
        for (int d = -3; d <= 3; d++) {
          const int i = Fh.i0 - NG + d;
          if (i < 0 || i >= ni) continue;
          nall--;
          if (i >= ilo && i <= iha && j >= jlo && j <= jhi && k >= klo && k <= khi) nint--;
        }
      }
    }
    // the fault planes deferred to the PLANE launch (welded nodes of the
    // grown split box; the split nodes belong to the fault kernels)
    if (s->pre_overlap)
      for (size_t f = 0; f < H.faults.size(); f++) {
        const FaultState &F = s->faults[f];
        const int i = H.faults[f].i0 - NG;
        if (i < ilo || i > iha || F.nj <= 0 || F.nk <= 0) continue;
        for (int k = std::max(klo, F.k0 - 3); k <= std::min(khi, F.k0 + F.nk + 2); k++)
          for (int j = std::max(jlo, F.j0 - 3); j <= std::min(jhi, F.j0 + F.nj + 2); j++)
            if (!(H.faults[f].flag[(size_t)(j + NG) + (size_t)(k + NG) * g.ny] & FL_SPLIT)) nint--;
      }
    s->int_points = nint;
    s->vol_points = nall;
  }
  CK(dalloc(s, &s->ctl, 1), "control block");
  for (int q = 0; q < 2; q++) CK(cudaEventCreate(&s->ev_run[q]), "event");
  for (int a = 0; a < 8; a++) for (int b = 0; b < 4; b++) for (int c = 0; c < 2; c++)
    CK(cudaEventCreate(&s->ev_vol[a][b][c]), "event");
  for (int a = 0; a < 8; a++) for (int b = 0; b < 4; b++) {
    CK(cudaEventCreate(&s->ev_int[a][b]), "event");
    CK(cudaEventCreate(&s->ev_int0[a][b]), "event");
  }
  {
    const char *br = std::getenv("CGFD_BRANCHES");
    if (br) s->branches = std::atoi(br);
    // the fault stream at the device's highest priority: the fault kernels
    // run beside whole-grid volume kernels, and their blocks should take
    // free SM slots first rather than wait for the volume grid's last wave
    // (CGFD_FAULT_PRIORITY=0: default priority)
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "stream priorities");
    const char *fp = std::getenv("CGFD_FAULT_PRIORITY");
    const bool hi = !(fp && fp[0] == '0');
    for (int q = 0; q < 3; q++)
      CK(cudaStreamCreateWithPriority(&s->aux[q], cudaStreamNonBlocking, q == 0 && hi ? prio_hi : prio_lo), "stream");
    for (int a = 0; a < 4; a++) {
      CK(cudaEventCreateWithFlags(&s->ev_stage[a], cudaEventDisableTiming), "event");
      CK(cudaEventCreateWithFlags(&s->ev_predone[a], cudaEventDisableTiming), "event");
      CK(cudaEventCreateWithFlags(&s->ev_postdone[a], cudaEventDisableTiming), "event");
      CK(cudaEventCreateWithFlags(&s->ev_fork[a], cudaEventDisableTiming), "event");
      CK(cudaEventCreateWithFlags(&s->ev_pre[a], cudaEventDisableTiming), "event");
      for (int b = 0; b < 3; b++) CK(cudaEventCreateWithFlags(&s->ev_join[a][b], cudaEventDisableTiming), "event");
    }
  }
  CK(cudaStreamSynchronize(s->stream), "set-up");
  {
    const char *tn = std::getenv("CGFD_TUNE");
    if (!std::getenv("CGFD_INTERIOR_YCHUNK") && !(tn && tn[0] == '0')) CK(tune_ychunk(s), "tuning");
  }
#undef CK
  {
    const int rc = build_graphs(s);
    if (rc != CGFD_OK) { destroy(s); return rc; }
  }
  *out = s;
  return CGFD_OK;
}

// capture step `it` (its operator pair it % 8, its level parity) into the
// graph of the current timing mode
static int build_graph(cgfd_solver *s, int it) {
  cudaGraphExec_t &G = s->graph[s->timing][it % 8];
  cudaGraph_t gr;
  cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(e, "begin capture");
  enqueue_step(s, it);
  // a launch refused during capture (bad configuration) is not part of the
  // graph and would otherwise go unnoticed
  const cudaError_t le = cudaGetLastError();
  e = cudaStreamEndCapture(s->stream, &gr);
  if (le != cudaSuccess) {
    if (e == cudaSuccess) cudaGraphDestroy(gr);
    return cuda_fail(le, "launch");
  }
  if (e != cudaSuccess) return cuda_fail(e, "end capture");
  e = cudaGraphInstantiate(&G, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) { G = nullptr; return cuda_fail(e, "instantiate"); }
  return CGFD_OK;
}

// the 8 step graphs of the current timing mode, built before any run so
// that no capture or instantiation happens between the launches of a run
static int build_graphs(cgfd_solver *s) {
  if (!s->use_graph) return CGFD_OK;
  for (int q = 0; q < 8; q++) {
    const int it = s->it + q;
    if (s->graph[s->timing][it % 8]) continue;
    const int rc = build_graph(s, it);
    if (rc != CGFD_OK) return rc;
  }
  return CGFD_OK;
}

int cgfd_run(cgfd_solver *s, int nsteps) {
  if (!s || nsteps < 0) return fail(CGFD_ERR_ARG, "bad argument");
  long long nl = 0;
  double vol_ms = 0, int_ms = 0;
  long long vol_n = 0, int_n = 0;
  const bool int_timed = s->nkbox[0] > 0;
  // with timing on, the events of step it (recorded by the graph of it % 8)
  // are read just before that graph is launched again 8 steps later, and
  // the last 8 after the loop: the host never waits on the step in flight
  auto read_events = [&](int it) -> cudaError_t {
    cudaError_t er = cudaEventSynchronize(s->ev_vol[it % 8][3][1]);
    if (er != cudaSuccess) return er;
    for (int st = 0; st < 4; st++) {
      float ms = 0;
      cudaEventElapsedTime(&ms, s->ev_vol[it % 8][st][0], s->ev_vol[it % 8][st][1]);
      vol_ms += ms;
      vol_n++;
      if (int_timed) {
        cudaEventElapsedTime(&ms, s->ev_int0[it % 8][st], s->ev_int[it % 8][st]);
        int_ms += ms;
        int_n++;
      }
    }
    return cudaSuccess;
  };
  const int it0 = s->it;
  cudaError_t e = cudaEventRecord(s->ev_run[0], s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "event");
  for (int q = 0; q < nsteps; q++) {
    const int it = s->it;
    if (s->timing && it - 8 >= it0) {
      e = read_events(it - 8);
      if (e != cudaSuccess) return cuda_fail(e, "timing");
    }
    if (s->use_graph) {
      cudaGraphExec_t &G = s->graph[s->timing][it % 8];
      if (!G) {
        const int rc = build_graph(s, it);
        if (rc != CGFD_OK) return rc;
      }
      e = cudaGraphLaunch(G, s->stream);
      if (e != cudaSuccess) return cuda_fail(e, "graph launch");
    } else {
      enqueue_step(s, it);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "launch");
    }
    nl += s->launches_per_step;
    s->it++;
  }
  e = cudaEventRecord(s->ev_run[1], s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "event");
  if (s->timing) {
    for (int it = std::max(it0, s->it - 8); it < s->it; it++) {
      e = read_events(it);
      if (e != cudaSuccess) return cuda_fail(e, "timing");
    }
  }
  s->last_launches = nl;
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "run");
  float run_ms = 0;
  cudaEventElapsedTime(&run_ms, s->ev_run[0], s->ev_run[1]);
  s->run_ms = run_ms; s->vol_ms = vol_ms; s->vol_launches = vol_n;
  s->int_ms = int_ms; s->int_launches = int_n;
  Ctl c;
  e = cudaMemcpy(&c, s->ctl, sizeof c, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "read control block");
  if (c.it != s->it) return fail(CGFD_ERR_STATE, "device step counter out of step with the host");
  if (c.err & CTL_ERR_NONFINITE) return fail(CGFD_ERR_UNSTABLE, "non-finite slip rate or station value");
  return CGFD_OK;
}

// ---- cgfd_run_fault_output ----------------------------------------------------

int cgfd_run_fault_output(cgfd_solver *s, int nsteps, int every, float *out, long long max_records, int *nrec) {
  if (!s || nsteps < 0 || every < 1 || max_records < 0) return fail(CGFD_ERR_ARG, "bad argument");
  const Grid &g = s->g;
  const int nf = (int)s->faults.size();
  const size_t fsz = (size_t)CGFD_FAULT_NFIELD * g.nj * g.nk, rsz = fsz * nf;
  long long want = 0;
  for (int q = 0; q < nsteps; q++) want += (s->it + q) % every == 0;
  if (want > max_records) return fail(CGFD_ERR_ARG, "output buffer holds fewer records than the run takes");
  if (want > 0 && (!out || nf == 0)) return fail(CGFD_ERR_ARG, "no output buffer, or no fault");
  if (nrec) *nrec = 0;
  cudaError_t e = cudaSuccess;
  if (want > 0 && !s->rec_buf[0]) {
    for (int b = 0; b < 2 && e == cudaSuccess; b++) e = dalloc(s, &s->rec_buf[b], rsz);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
      e = cudaEventCreateWithFlags(&s->ev_gathered[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_copied[b], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return cuda_fail(e, "fault output staging");
  }
  long long nl = 0, rec = 0;
  e = cudaEventRecord(s->ev_run[0], s->stream);
  for (int q = 0; q < nsteps && e == cudaSuccess; q++) {
    const int it = s->it;
    if (it % every == 0) {
      // gather into the staging buffer of this record's parity once its
      // previous copy has left it, then copy it out on the copy stream
      // while the next steps run
      const int b = (int)(rec & 1);
      if (rec >= 2) e = cudaStreamWaitEvent(s->stream, s->ev_copied[b], 0);
      for (int f = 0; f < nf && e == cudaSuccess; f++) {
        launch_fault_gather(s->faults[f].out, s->rec_buf[b] + f * fsz, CGFD_FAULT_NFIELD, g, s->stream);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaEventRecord(s->ev_gathered[b], s->stream);
#ifdef CGFD_FP64
      if (e == cudaSuccess) e = to_host(out + rec * rsz, s->rec_buf[b], rsz, s->stream);
#else
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy, s->ev_gathered[b], 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(out + rec * rsz, s->rec_buf[b], rsz * sizeof(real), cudaMemcpyDeviceToHost, s->copy);
      if (e == cudaSuccess) e = cudaEventRecord(s->ev_copied[b], s->copy);
#endif
      rec++;
      nl += nf;
    }
    if (e != cudaSuccess) break;
    if (s->use_graph) {
      cudaGraphExec_t &G = s->graph[s->timing][it % 8];
      if (!G) {
        const int rc = build_graph(s, it);
        if (rc != CGFD_OK) return rc;
      }
      e = cudaGraphLaunch(G, s->stream);
    } else {
      enqueue_step(s, it);
      e = cudaGetLastError();
    }
    nl += s->launches_per_step;
    s->it++;
  }
  if (e == cudaSuccess) e = cudaEventRecord(s->ev_run[1], s->stream);
  if (e == cudaSuccess && s->copy) e = cudaStreamSynchronize(s->copy);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "run with fault output");
  if (nrec) *nrec = (int)rec;
  float run_ms = 0;
  cudaEventElapsedTime(&run_ms, s->ev_run[0], s->ev_run[1]);
  s->run_ms = run_ms; s->vol_ms = s->int_ms = 0; s->vol_launches = s->int_launches = 0;
  s->last_launches = nl;
  Ctl c;
  e = cudaMemcpy(&c, s->ctl, sizeof c, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "read control block");
  if (c.it != s->it) return fail(CGFD_ERR_STATE, "device step counter out of step with the host");
  if (c.err & CTL_ERR_NONFINITE) return fail(CGFD_ERR_UNSTABLE, "non-finite slip rate or station value");
  return CGFD_OK;
}

int cgfd_host_alloc(unsigned long long bytes, void **ptr) {
  if (!ptr) return fail(CGFD_ERR_ARG, "bad argument");
  *ptr = nullptr;
  const cudaError_t e = cudaMallocHost(ptr, std::max<unsigned long long>(bytes, 1));
  if (e != cudaSuccess) { *ptr = nullptr; return cuda_fail(e, "page-locked host memory"); }
  return CGFD_OK;
}

void cgfd_host_free(void *ptr) {
  if (ptr) cudaFreeHost(ptr);
}

// ---- cgfd_run_noalloc ------------------------------------------------------

namespace {
constexpr int kNoallocMaxDevices = 64;
std::atomic<real *> g_noalloc_ptr[kNoallocMaxDevices];

int fail_fixed(int code, const char *m) {
  size_t n = 0;
  for (; m[n] && n + 1 < sizeof g_err_fixed; n++) g_err_fixed[n] = m[n];
  g_err_fixed[n] = 0;
  g_err_is_fixed = true;
  return code;
}

int fail_fixed_cuda(cudaError_t e, const char *what) {
  char b[sizeof g_err_fixed];
  std::snprintf(b, sizeof b, "%s: %s", what, cudaGetErrorString(e));
  return fail_fixed(e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA, b);
}
}  // namespace

int cgfd_run_noalloc(cgfd_solver *s, int nsteps) {
  if (!s || nsteps < 0) return fail_fixed(CGFD_ERR_ARG, "bad argument");
  // every fault takes its own slice of the static array: their sum must fit
  size_t toff[MAXF];
  const unsigned long long need = trac_slices(s, toff);
  if (need > CGFD_NOALLOC_SCRATCH_FLOATS) {
    char b[sizeof g_err_fixed];
    std::snprintf(b, sizeof b,
                  "cgfd_run_noalloc: the faults' split boxes need %llu scratch floats together, the static array holds %u",
                  need, CGFD_NOALLOC_SCRATCH_FLOATS);
    return fail_fixed(CGFD_ERR_ARG, b);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_fixed_cuda(e, "cgfd_run_noalloc: current device");
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail_fixed(CGFD_ERR_ARG, "cgfd_run_noalloc: device ordinal too large");
  real *trac = g_noalloc_ptr[dev].load();
  if (!trac) {
    e = noalloc_scratch_address(&trac);
    if (e != cudaSuccess) return fail_fixed_cuda(e, "cgfd_run_noalloc: scratch address");
    g_noalloc_ptr[dev].store(trac);
  }
  long long nl = 0;
  s->run_ms = s->vol_ms = s->int_ms = 0;
  s->vol_launches = s->int_launches = 0;
  for (int q = 0; q < nsteps; q++) {
    enqueue_step(s, s->it, trac, false);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_fixed_cuda(e, "cgfd_run_noalloc: launch");
    nl += s->launches_per_step;
    s->it++;
  }
  s->last_launches = nl;
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return fail_fixed_cuda(e, "cgfd_run_noalloc: run");
  Ctl c;
  e = cudaMemcpy(&c, s->ctl, sizeof c, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail_fixed_cuda(e, "cgfd_run_noalloc: read control block");
  if (c.it != s->it) return fail_fixed(CGFD_ERR_STATE, "device step counter out of step with the host");
  if (c.err & CTL_ERR_NONFINITE) return fail_fixed(CGFD_ERR_UNSTABLE, "non-finite slip rate or station value");
  return CGFD_OK;
}

// ---- ensembles ---------------------------------------------------------------
struct cgfd_ensemble {
  std::vector<cgfd_solver *> m;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph[8] = {};
};

static void ensemble_free(cgfd_ensemble *e) {
  if (!e) return;
  for (int q = 0; q < 8; q++) if (e->graph[q]) cudaGraphExecDestroy(e->graph[q]);
  for (cudaEvent_t ev : e->join) if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->origin) cudaStreamDestroy(e->origin);
  delete e;
}

int cgfd_ensemble_create(cgfd_solver *const *members, int n, cgfd_ensemble **out) {
  if (!members || n <= 0 || !out) return fail(CGFD_ERR_ARG, "bad argument");
  *out = nullptr;
  for (int q = 0; q < n; q++) {
    if (!members[q]) return fail(CGFD_ERR_ARG, "null ensemble member");
    if (members[q]->it != members[0]->it) return fail(CGFD_ERR_STATE, "ensemble members at different steps");
    for (int r = 0; r < q; r++)
      if (members[r] == members[q]) return fail(CGFD_ERR_ARG, "solver given twice to an ensemble");
  }
  cgfd_ensemble *e = new cgfd_ensemble();
  e->m.assign(members, members + n);
  cudaError_t er = cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking);
  if (er == cudaSuccess) er = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
  e->join.assign(n, nullptr);
  for (int q = 0; q < n && er == cudaSuccess; q++) er = cudaEventCreateWithFlags(&e->join[q], cudaEventDisableTiming);
  if (er != cudaSuccess) { ensemble_free(e); return cuda_fail(er, "ensemble set-up"); }
  *out = e;
  return CGFD_OK;
}

int cgfd_ensemble_run(cgfd_ensemble *e, int nsteps) {
  if (!e || nsteps < 0) return fail(CGFD_ERR_ARG, "bad argument");
  const int n = (int)e->m.size();
  for (int q = 1; q < n; q++)
    if (e->m[q]->it != e->m[0]->it) return fail(CGFD_ERR_STATE, "ensemble members out of step (cgfd_run on a member?)");
  cudaError_t er;
  for (int step = 0; step < nsteps; step++) {
    const int it = e->m[0]->it;
    cudaGraphExec_t &G = e->graph[it % 8];
    if (!G) {
      // fork from the origin stream to every member's stream, one step of
      // each member, join back: a graph with one branch per member
      cudaGraph_t gr;
      er = cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal);
      if (er != cudaSuccess) return cuda_fail(er, "begin ensemble capture");
      cudaEventRecord(e->fork, e->origin);
      for (int q = 0; q < n; q++) {
        cgfd_solver *s = e->m[q];
        cudaStreamWaitEvent(s->stream, e->fork, 0);
        // beside the other members each member's step runs best with the y
        // / z PML slabs on its main stream and the fault slab kernels after
        // its interior kernel (measured: +2% over the solo default); the
        // schedules change no arithmetic
        const int br0 = s->branches;
        const bool pe0 = s->post_early;
        if (s->branches == 3) s->branches = 2;
        s->post_early = false;
        enqueue_step(s, it, nullptr, false);
        s->branches = br0;
        s->post_early = pe0;
        cudaEventRecord(e->join[q], s->stream);
        cudaStreamWaitEvent(e->origin, e->join[q], 0);
      }
      const cudaError_t le = cudaGetLastError();
      er = cudaStreamEndCapture(e->origin, &gr);
      if (le != cudaSuccess) {
        if (er == cudaSuccess) cudaGraphDestroy(gr);
        return cuda_fail(le, "ensemble launch");
      }
      if (er != cudaSuccess) return cuda_fail(er, "end ensemble capture");
      er = cudaGraphInstantiate(&G, gr, 0);
      cudaGraphDestroy(gr);
      if (er != cudaSuccess) { G = nullptr; return cuda_fail(er, "instantiate ensemble graph"); }
    }
    er = cudaGraphLaunch(G, e->origin);
    if (er != cudaSuccess) return cuda_fail(er, "ensemble graph launch");
    for (cgfd_solver *s : e->m) { s->it++; s->last_launches = 0; }
  }
  er = cudaStreamSynchronize(e->origin);
  if (er != cudaSuccess) return cuda_fail(er, "ensemble run");
  for (int q = 0; q < n; q++) {
    cgfd_solver *s = e->m[q];
    s->last_launches = (long long)nsteps * s->launches_per_step;
    Ctl c;
    er = cudaMemcpy(&c, s->ctl, sizeof c, cudaMemcpyDeviceToHost);
    if (er != cudaSuccess) return cuda_fail(er, "read control block");
    const std::string who = "ensemble member " + std::to_string(q) + ": ";
    if (c.it != s->it) return fail(CGFD_ERR_STATE, who + "device step counter out of step with the host");
    if (c.err & CTL_ERR_NONFINITE) return fail(CGFD_ERR_UNSTABLE, who + "non-finite slip rate or station value");
  }
  return CGFD_OK;
}

void cgfd_ensemble_destroy(cgfd_ensemble *e) { ensemble_free(e); }

int cgfd_set_timing(cgfd_solver *s, int on) {
  if (!s) return fail(CGFD_ERR_ARG, "bad argument");
  s->timing = on ? 1 : 0;
  return build_graphs(s);
}

int cgfd_last_timing(const cgfd_solver *s, double *run_ms, double *volume_ms, long long *volume_launches) {
  if (!s) return fail(CGFD_ERR_ARG, "bad argument");
  if (run_ms) *run_ms = s->run_ms;
  if (volume_ms) *volume_ms = s->vol_ms;
  if (volume_launches) *volume_launches = s->vol_launches;
  return CGFD_OK;
}

int cgfd_last_kernel_timing(const cgfd_solver *s, int which, double *ms, long long *launches, long long *points) {
  if (!s || which < 0 || which > 1) return fail(CGFD_ERR_ARG, "bad argument");
  if (ms) *ms = which ? s->int_ms : s->vol_ms;
  if (launches) *launches = which ? s->int_launches : s->vol_launches;
  if (points) *points = which ? s->int_points : s->vol_points;
  return CGFD_OK;
}

int cgfd_steps_done(const cgfd_solver *s, int *it) {
  if (!s || !it) return fail(CGFD_ERR_ARG, "bad argument");
  *it = s->it;
  return CGFD_OK;
}

int cgfd_dt_max(const cgfd_solver *s, float *d) {
  if (!s || !d) return fail(CGFD_ERR_ARG, "bad argument");
  *d = s->dtmax;
  return CGFD_OK;
}

int cgfd_get_fault_all(cgfd_solver *s, int f, float *out) {
  if (!s || !out || f < 0 || f >= (int)s->faults.size()) return fail(CGFD_ERR_ARG, "bad argument");
  const Grid &g = s->g;
  // gather the interior nodes on the device, then one contiguous copy
  launch_fault_gather(s->faults[f].out, s->faults[f].gather, CGFD_FAULT_NFIELD, g, s->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = to_host(out, s->faults[f].gather, (size_t)CGFD_FAULT_NFIELD * g.nj * g.nk, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "read fault");
  return CGFD_OK;
}

int cgfd_get_fault(cgfd_solver *s, int f, int field, float *out) {
  if (!s || !out || f < 0 || f >= (int)s->faults.size() || field < 0 || field >= CGFD_FAULT_NFIELD)
    return fail(CGFD_ERR_ARG, "bad argument");
  const Grid &g = s->g;
  const size_t ns = (size_t)g.ny * g.nz;
  std::vector<float> h(ns);
  cudaError_t e = to_host(h.data(), s->faults[f].out + field * ns, ns, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "read fault");
  for (int k = 0; k < g.nk; k++) std::memcpy(out + (size_t)k * g.nj, h.data() + (size_t)(k + NG) * g.ny + NG, (size_t)g.nj * 4);
  return CGFD_OK;
}

static int get_series(cgfd_solver *s, real *dev, int n, float *out, int *nrec) {
  Ctl c;
  cudaError_t e = cudaMemcpy(&c, s->ctl, sizeof c, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "read control block");
  if (nrec) *nrec = c.nrec;
  if (!out || n == 0 || c.nrec == 0) return CGFD_OK;
  const int mr = s->st.max_rec;
  std::vector<float> h((size_t)n * 9 * mr);
  e = to_host(h.data(), dev, h.size(), s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "read series");
  for (size_t q = 0; q < (size_t)n * 9; q++) std::memcpy(out + q * c.nrec, h.data() + q * mr, (size_t)c.nrec * 4);
  return CGFD_OK;
}

int cgfd_get_stations(cgfd_solver *s, float *out, int *nrec) {
  if (!s) return fail(CGFD_ERR_ARG, "bad argument");
  return get_series(s, s->seis, s->st.n, out, nrec);
}

int cgfd_get_fault_stations(cgfd_solver *s, float *out, int *nrec) {
  if (!s) return fail(CGFD_ERR_ARG, "bad argument");
  return get_series(s, s->fseis, s->st.nf, out, nrec);
}

// the array of one level that holds component cmp: the 16-byte groups
// (Vx Vy Vz Txx), (Tyy Tzz Tyz Txz) or Txy; element of point p at
// p * step + lane
struct CmpArray { size_t off, n; int step, lane; };
static CmpArray cmp_array(const Grid &g, int cmp) {
  const size_t sc = g.scmp;
  if (cmp < 4) return { 0, 4 * sc, 4, cmp };
  if (cmp < 8) return { 4 * sc, 4 * sc, 4, cmp - 4 };
  return { 8 * sc, sc, 1, 0 };
}

int cgfd_get_surface_peaks(cgfd_solver *s, float *out) {
  if (!s || !out) return fail(CGFD_ERR_ARG, "bad argument");
  if (!s->pg) return fail(CGFD_ERR_ARG, "no free surface: no surface peaks");
  const size_t n = (size_t)CGFD_NPEAK * s->g.ni * s->g.nj;
  cudaError_t e = to_host(out, s->pg, n, s->stream);
  return e == cudaSuccess ? CGFD_OK : cuda_fail(e, "read surface peaks");
}

int cgfd_get_wavefield(cgfd_solver *s, int cmp, float *out) {
  if (!s || !out || cmp < 0 || cmp >= NCMP) return fail(CGFD_ERR_ARG, "bad argument");
  const Grid &g = s->g;
  const CmpArray A = cmp_array(g, cmp);
  std::vector<float> h(A.n);
  cudaError_t e = to_host(h.data(), s->w[slot(LP, s->it)] + A.off, A.n, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "read wavefield");
  for (int k = 0; k < g.nk; k++)
    for (int j = 0; j < g.nj; j++) {
      const float *src = h.data() + (size_t)g.at(NG, j + NG, k + NG) * A.step + A.lane;
      float *dst = out + ((size_t)k * g.nj + j) * g.ni;
      for (int i = 0; i < g.ni; i++) dst[i] = src[(size_t)i * A.step];
    }
  return CGFD_OK;
}

int cgfd_set_wavefield(cgfd_solver *s, int cmp, const float *in) {
  if (!s || !in || cmp < 0 || cmp >= NCMP) return fail(CGFD_ERR_ARG, "bad argument");
  const Grid &g = s->g;
  const CmpArray A = cmp_array(g, cmp);
  std::vector<float> h(A.n);
  real *dst = s->w[slot(LP, s->it)] + A.off;
  cudaError_t e = to_host(h.data(), dst, A.n, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "read wavefield");
  for (int k = 0; k < g.nk; k++)
    for (int j = 0; j < g.nj; j++) {
      float *d = h.data() + (size_t)g.at(NG, j + NG, k + NG) * A.step + A.lane;
      const float *src = in + ((size_t)k * g.nj + j) * g.ni;
      for (int i = 0; i < g.ni; i++) d[(size_t)i * A.step] = src[i];
    }
  e = to_device(dst, h.data(), A.n, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "write wavefield");
  return CGFD_OK;
}

// checkpoint: [Ctl][P level][PML P levels][per fault: P level, scal, out, flag][seis][fseis]
// [surface peaks, surface displacement (free surface only)]
static std::vector<std::pair<void *, size_t>> state_parts(cgfd_solver *s) {
  std::vector<std::pair<void *, size_t>> v;
  const Grid &g = s->g;
  const size_t ns = (size_t)g.ny * g.nz;
  const int sp = slot(LP, s->it);
  v.push_back({ s->ctl, sizeof(Ctl) });
  v.push_back({ s->w[sp], (size_t)NCMP * g.scmp * sizeof(real) });
  for (int q = 0; q < 6; q++) if (s->pml[q].d.on) v.push_back({ s->pml[q].aux[sp], (size_t)NCMP * s->pml[q].d.siz * sizeof(real) });
  for (auto &F : s->faults) {
    v.push_back({ F.lev[sp], 18 * ns * sizeof(real) });
    v.push_back({ F.scal, (size_t)NFS * ns * sizeof(real) });
    v.push_back({ F.out, (size_t)CGFD_FAULT_NFIELD * ns * sizeof(real) });
    v.push_back({ F.flag, ns });
  }
  v.push_back({ s->seis, (size_t)s->st.n * 9 * std::max(1, s->st.max_rec) * sizeof(real) });
  v.push_back({ s->fseis, (size_t)s->st.nf * 9 * std::max(1, s->st.max_rec) * sizeof(real) });
  if (s->pg) {
    v.push_back({ s->pg, (size_t)CGFD_NPEAK * g.ni * g.nj * sizeof(real) });
    v.push_back({ s->dis, (size_t)3 * g.ni * g.nj * sizeof(real) });
  }
  return v;
}

int cgfd_checkpoint_size(cgfd_solver *s, unsigned long long *bytes) {
  if (!s || !bytes) return fail(CGFD_ERR_ARG, "bad argument");
  unsigned long long n = sizeof(int);
  for (auto &p : state_parts(s)) n += p.second;
  *bytes = n;
  return CGFD_OK;
}

int cgfd_checkpoint(cgfd_solver *s, void *buf, unsigned long long bytes) {
  unsigned long long need = 0;
  int rc = cgfd_checkpoint_size(s, &need);
  if (rc) return rc;
  if (!buf || bytes < need) return fail(CGFD_ERR_ARG, "checkpoint buffer too small");
  char *p = (char *)buf;
  std::memcpy(p, &s->it, sizeof(int));
  p += sizeof(int);
  for (auto &q : state_parts(s)) {
    cudaError_t e = cudaMemcpy(p, q.first, q.second, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "checkpoint");
    p += q.second;
  }
  return CGFD_OK;
}

int cgfd_restore(cgfd_solver *s, const void *buf, unsigned long long bytes) {
  unsigned long long need = 0;
  int rc = cgfd_checkpoint_size(s, &need);
  if (rc) return rc;
  if (!buf || bytes != need) return fail(CGFD_ERR_ARG, "checkpoint size does not match this solver");
  const char *p = (const char *)buf;
  int it;
  std::memcpy(&it, p, sizeof(int));
  p += sizeof(int);
  if (it < 0) return fail(CGFD_ERR_ARG, "corrupt checkpoint");
  s->it = it;   // sets the level parity before the parts are placed
  for (auto &q : state_parts(s)) {
    cudaError_t e = cudaMemcpy(q.first, p, q.second, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "restore");
    p += q.second;
  }
  return CGFD_OK;
}

int cgfd_last_launches(const cgfd_solver *s, long long *n) {
  if (!s || !n) return fail(CGFD_ERR_ARG, "bad argument");
  *n = s->last_launches;
  return CGFD_OK;
}

void cgfd_destroy(cgfd_solver *s) {
  if (s) cudaStreamSynchronize(s->stream);
  destroy(s);
}

}  // extern "C"
