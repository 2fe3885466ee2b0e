// cgfd_run.cpp -- command-line forward run from the reference's parameter
// file, on one B200.
//
//     cgfd_run par.json [gpu_id]
//     cgfd_run --check par.json     (inputs and host set-up only, no GPU)
//
// Replaces `main par.json gpu_id_start` (src/forward/main_curv_col_el_3d.cu)
// for one GPU: the same par keys (src/forward/par_t.cu:64-720), the same
// input files (fault_coord_<id>.nc, init_stress_<id>.nc, coord_px0_py0_pz0.nc,
// media_px0_py0_pz0.nc, the station and fault-station lists) and the same
// outputs in output_dir:
//   fault_i<x>_px0_py0_pz0.nc   time, Tn .. Slip2 every io_time_skip steps,
//                               Peak_vs and Init_t0 at the end
//                               (io_funcs.cu:1911-2164)
//   <station>.<Vx..Txy>.sac     station seismograms (io_funcs.cu:578-617)
//   fault_<station>.<Tn..Slip2>.sac  fault stations (io_funcs.cu:2355-2400)
//   <station>.<Exx..Exy>.sac    strain at the stations (io_funcs.cu:620-700)
//   PG_V_A_D_px0_py0_pz0.nc     peak surface velocity, acceleration and
//                               displacement with a free surface
//                               (io_funcs.cu:1827-1880)
// The time stepping runs in libcgfd (include/cgfd.h).  Par keys of outputs
// outside the forward path (receiver_line, slice, snapshot, grid / metric /
// media export), keys without effect on one GPU and keys the reference does
// not read either are reported on stderr and ignored.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cgfd.h"
#include "json.h"
#include "ncclassic.h"
#include "sac.h"

using cgfd_json::Value;

namespace {

[[noreturn]] void die(const std::string &m) {
  std::fprintf(stderr, "cgfd_run: %s\n", m.c_str());
  std::exit(1);
}

void check(int rc, const char *what) {
  if (rc != CGFD_OK) die(std::string(what) + ": " + cgfd_last_error());
}

std::string read_file(const std::string &path) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

double num(const Value &root, const char *key, double dflt) {
  const Value *v = root.get(key);
  return v && v->kind == Value::Number ? v->num : dflt;
}
std::string str(const Value &root, const char *key, const std::string &dflt = "") {
  const Value *v = root.get(key);
  return v && v->kind == Value::String ? v->str : dflt;
}

// next line that is neither empty nor a comment (io_get_nextline,
// io_funcs.cu:1886-1908)
bool next_line(std::ifstream &f, std::string &line) {
  while (std::getline(f, line)) {
    if (!line.empty() && line[0] != '#' && line[0] != '\r') return true;
  }
  return false;
}

struct Station {
  std::string name;
  float i, j, k;        // 0-based fractional grid indices
};
struct FaultStation {
  std::string name;
  int fault;
  float j, k;
};

// 2-D [nk][nj] variable of a classic file
std::vector<float> read_plane(const cgfd_nc::Reader &r, const std::string &name, int nj, int nk,
                              const std::string &file) {
  const int v = r.var(name);
  if (v < 0) die(file + ": no variable " + name);
  std::vector<float> out((size_t)nj * nk);
  r.get_float(v, { 0, 0 }, { (size_t)nk, (size_t)nj }, out.data());
  return out;
}
std::vector<float> read_volume(const cgfd_nc::Reader &r, const std::string &name, int ni, int nj, int nk,
                               const std::string &file) {
  const int v = r.var(name);
  if (v < 0) die(file + ": no variable " + name);
  std::vector<float> out((size_t)ni * nj * nk);
  r.get_float(v, { 0, 0, 0 }, { (size_t)nk, (size_t)nj, (size_t)ni }, out.data());
  return out;
}

}  // namespace

// How the driver treats each top-level key of the reference's par file
// (par_t.cu:64-900 reads them with cJSON, which ignores any other key).
enum KeyUse { KEY_USED, KEY_NO_OUTPUT, KEY_NO_EFFECT };
const struct { const char *key; KeyUse use; } kParKeys[] = {
  { "number_of_total_grid_points_x", KEY_USED }, { "number_of_total_grid_points_y", KEY_USED },
  { "number_of_total_grid_points_z", KEY_USED }, { "size_of_time_step", KEY_USED },
  { "number_of_time_steps", KEY_USED }, { "time_window_length", KEY_USED }, { "time_start", KEY_USED },
  { "time_check_stability", KEY_USED }, { "io_time_skip", KEY_USED }, { "dynamic_method", KEY_USED },
  { "fault_x_index", KEY_USED }, { "fault_grid", KEY_USED }, { "boundary_x_left", KEY_USED },
  { "boundary_x_right", KEY_USED }, { "boundary_y_front", KEY_USED }, { "boundary_y_back", KEY_USED },
  { "boundary_z_bottom", KEY_USED }, { "boundary_z_top", KEY_USED }, { "grid_generation_method", KEY_USED },
  { "metric_calculation_method", KEY_USED }, { "medium", KEY_USED }, { "output_dir", KEY_USED },
  { "in_station_file", KEY_USED }, { "fault_station_file", KEY_USED }, { "welded_margin", KEY_USED },
  // outputs outside the forward path's fault and station files
  { "receiver_line", KEY_NO_OUTPUT }, { "slice", KEY_NO_OUTPUT }, { "snapshot", KEY_NO_OUTPUT },
  { "is_export_grid", KEY_NO_OUTPUT }, { "grid_export_dir", KEY_NO_OUTPUT }, { "is_export_metric", KEY_NO_OUTPUT },
  { "is_export_media", KEY_NO_OUTPUT }, { "media_export_dir", KEY_NO_OUTPUT }, { "output_all", KEY_NO_OUTPUT },
  // no effect with the whole domain on one GPU, or only a message in the reference
  { "number_of_mpiprocs_x", KEY_NO_EFFECT }, { "number_of_mpiprocs_y", KEY_NO_EFFECT },
  { "number_of_mpiprocs_z", KEY_NO_EFFECT }, { "check_nan_every_number_of_steps", KEY_NO_EFFECT },
  { "visco_config", KEY_NO_EFFECT },
};

// one line per top-level key that does not change the run: outputs this
// driver does not write, keys without effect on one GPU, and keys the
// reference does not read either (cJSON skips them: a leading '#' is the
// examples' way of commenting a key out; misspelt keys fall here too)
void report_keys(const Value &par) {
  for (const auto &kv : par.obj) {
    const std::string &k = kv.first;
    int use = -1;
    for (const auto &e : kParKeys) if (k == e.key) use = e.use;
    if (use == KEY_USED) continue;
    if (use == KEY_NO_OUTPUT)
      std::fprintf(stderr, "cgfd_run: %s: output not produced by this driver, ignored\n", k.c_str());
    else if (use == KEY_NO_EFFECT)
      std::fprintf(stderr, "cgfd_run: %s: no effect on a single-GPU run, ignored\n", k.c_str());
    else if (!k.empty() && k[0] == '#')
      std::fprintf(stderr, "cgfd_run: %s: commented out, ignored\n", k.c_str());
    else
      std::fprintf(stderr, "cgfd_run: %s: not a key of the reference's par file, ignored\n", k.c_str());
  }
}

int main(int argc, char **argv) {
  // --check: parse the par file, read every input file and run the host
  // set-up (grid, metric, medium, PML, fault coefficients), then report the
  // configuration and exit; needs no GPU
  bool check_only = false;
  if (argc > 1 && std::strcmp(argv[1], "--check") == 0) {
    check_only = true;
    argv++;
    argc--;
  }
  if (argc < 2) die("usage: cgfd_run [--check] par.json [gpu_id]");
  const int gpu = argc > 2 ? std::atoi(argv[2]) : 0;
  Value par;
  try {
    par = cgfd_json::parse(read_file(argv[1]));
  } catch (const std::exception &e) {
    die(e.what());
  }
  if (par.kind != Value::Object) die("par file: a JSON object expected");
  report_keys(par);

  // ---- grid, time ---------------------------------------------------------
  cgfd_config cfg;
  cgfd_config_default(&cfg);
  cfg.ni = (int)num(par, "number_of_total_grid_points_x", 0);
  cfg.nj = (int)num(par, "number_of_total_grid_points_y", 0);
  cfg.nk = (int)num(par, "number_of_total_grid_points_z", 0);
  if (cfg.ni <= 0 || cfg.nj <= 0 || cfg.nk <= 0) die("number_of_total_grid_points_{x,y,z} missing");
  const int ni = cfg.ni, nj = cfg.nj, nk = cfg.nk;
  if (num(par, "number_of_mpiprocs_y", 1) != 1 || num(par, "number_of_mpiprocs_z", 1) != 1)
    std::fprintf(stderr, "cgfd_run: number_of_mpiprocs_* ignored: the whole domain runs on one GPU\n");
  const double dt = num(par, "size_of_time_step", -1.0);
  int nt = (int)num(par, "number_of_time_steps", -1);
  const double twin = num(par, "time_window_length", -1.0);
  if (dt <= 0.0) die("size_of_time_step missing");
  if (nt < 0) {
    if (twin < 0.0) die("number_of_time_steps or time_window_length needed");
    nt = (int)(twin / dt + 0.5);
  }
  // the reference's time loop takes number_of_time_steps + 1 steps
  // (nt_total, main_curv_col_el_3d.cu:483; drv_rk_curv_col.cu:209)
  const int nt_total = nt + 1;
  const double t0 = num(par, "time_start", 0.0);
  const int skip = std::max(1, (int)num(par, "io_time_skip", 1));
  cfg.dt = (float)dt;
  cfg.check_stability = (int)num(par, "time_check_stability", 1);
  cfg.dynamic_method = (int)num(par, "dynamic_method", 2);
  // not a key of the reference, whose margin of welded nodes is fixed at 40
  // (fault_info.cu:1044-1060); lets small test grids keep split nodes
  cfg.welded_margin = (int)num(par, "welded_margin", 40);

  // ---- faults -------------------------------------------------------------
  const Value *fx = par.get("fault_x_index");
  const Value *fg = par.get("fault_grid");
  if (!fx || fx->kind != Value::Array || fx->arr.empty()) die("fault_x_index missing");
  cfg.num_faults = (int)fx->arr.size();
  if (cfg.num_faults > CGFD_MAX_FAULTS) die("too many faults");
  if (!fg || fg->kind != Value::Array || (int)fg->arr.size() < 4 * cfg.num_faults) die("fault_grid missing");
  for (int f = 0; f < cfg.num_faults; f++) {
    cfg.fault_x_index[f] = fx->arr[f].as_int();
    for (int q = 0; q < 4; q++) cfg.fault_grid[f][q] = fg->arr[4 * f + q].as_int();
  }

  // ---- boundaries (par_t.cu:160-312) --------------------------------------
  const char *bnames[3][2] = { { "boundary_x_left", "boundary_x_right" }, { "boundary_y_front", "boundary_y_back" },
                               { "boundary_z_bottom", "boundary_z_top" } };
  for (int d = 0; d < 3; d++)
    for (int s = 0; s < 2; s++) {
      const Value *b = par.get(bnames[d][s]);
      if (!b) continue;
      if (const Value *p = b->get("cfspml")) {
        cfg.pml_layers[d][s] = (int)num(*p, "number_of_layers", 0);
        cfg.pml_alpha_max[d][s] = (float)num(*p, "alpha_max", 0.0);
        cfg.pml_beta_max[d][s] = (float)num(*p, "beta_max", 1.0);
        cfg.pml_ref_vel[d][s] = (float)num(*p, "ref_vel", 0.0);
      }
      if (const Value *p = b->get("ablexp")) {
        cfg.ablexp_layers[d][s] = (int)num(*p, "number_of_layers", 0);
        cfg.ablexp_ref_vel[d][s] = (float)num(*p, "ref_vel", 0.0);
      }
      if (d == 2 && s == 1 && b->get("free")) cfg.free_surface = 1;
    }

  // ---- geometry -----------------------------------------------------------
  std::vector<std::vector<float>> keep;   // arrays the config points into
  auto hold = [&](std::vector<float> v) { keep.push_back(std::move(v)); return keep.back().data(); };
  const Value *gm = par.get("grid_generation_method");
  if (!gm) die("grid_generation_method missing");
  std::string stress_dir;
  try {
    if (const Value *fp = gm->get("fault_plane")) {
      cfg.grid_mode = CGFD_GRID_FAULT_PLANE;
      const std::string dir = str(*fp, "fault_geometry_dir");
      stress_dir = str(*fp, "fault_init_stress_dir");
      cfg.fault_interval = (float)num(*fp, "fault_inteval", 0.0);
      std::vector<float> X, Y, Z;
      for (int f = 0; f < cfg.num_faults; f++) {
        const std::string file = dir + "/fault_coord_" + std::to_string(f + 1) + ".nc";
        cgfd_nc::Reader r(file);
        const std::vector<float> x = read_plane(r, "x", nj, nk, file), y = read_plane(r, "y", nj, nk, file),
                                 z = read_plane(r, "z", nj, nk, file);
        X.insert(X.end(), x.begin(), x.end()); Y.insert(Y.end(), y.begin(), y.end()); Z.insert(Z.end(), z.begin(), z.end());
      }
      cfg.fault_x = hold(X); cfg.fault_y = hold(Y); cfg.fault_z = hold(Z);
    } else if (const Value *gi = gm->get("grid_import")) {
      cfg.grid_mode = CGFD_GRID_IMPORT;
      stress_dir = str(*gi, "fault_init_stress_dir");
      const std::string file = str(*gi, "import_dir") + "/coord_px0_py0_pz0.nc";
      cgfd_nc::Reader r(file);
      cfg.x3d = hold(read_volume(r, "x", ni, nj, nk, file));
      cfg.y3d = hold(read_volume(r, "y", ni, nj, nk, file));
      cfg.z3d = hold(read_volume(r, "z", ni, nj, nk, file));
    } else {
      die("grid_generation_method: fault_plane or grid_import expected");
    }

    // ---- medium (md_gen_uniform_el_iso, md_t.cu:378-417; md_import, :230-288)
    const Value *md = par.get("medium");
    const std::string way = md ? str(*md, "input_way", "code") : "code";
    if (md && str(*md, "type", "elastic_iso") != "elastic_iso") die("medium: only elastic_iso is supported");
    const size_t np = (size_t)ni * nj * nk;
    if (way == "code") {
      const float vp = 6000.0f, vs = 3464.0f, rho = 2670.0f;
      // float products, the subtraction in double (2.0 is a double literal there)
      const float mu = vs * vs * rho;
      const float lam = (float)((double)(vp * vp * rho) - 2.0 * (double)mu);
      cfg.lambda = hold(std::vector<float>(np, lam));
      cfg.mu = hold(std::vector<float>(np, mu));
      cfg.rho = hold(std::vector<float>(np, rho));
    } else if (way == "import") {
      const std::string file = str(*md, "import") + "/media_px0_py0_pz0.nc";
      cgfd_nc::Reader r(file);
      cfg.lambda = hold(read_volume(r, "lambda", ni, nj, nk, file));
      cfg.mu = hold(read_volume(r, "mu", ni, nj, nk, file));
      cfg.rho = hold(read_volume(r, "rho", ni, nj, nk, file));
    } else {
      die("medium input_way " + way + " is not supported (code or import)");
    }

    // ---- initial stress and friction (fault_info.cu:1077-1187) -------------
    std::vector<float> T[7];
    const char *snames[7] = { "Tx", "Ty", "Tz", "mu_s", "mu_d", "Dc", "C0" };
    for (int f = 0; f < cfg.num_faults; f++) {
      const std::string file = stress_dir + "/init_stress_" + std::to_string(f + 1) + ".nc";
      cgfd_nc::Reader r(file);
      for (int q = 0; q < 7; q++) {
        const std::vector<float> v = read_plane(r, snames[q], nj, nk, file);
        T[q].insert(T[q].end(), v.begin(), v.end());
      }
    }
    cfg.T0x = hold(T[0]); cfg.T0y = hold(T[1]); cfg.T0z = hold(T[2]);
    cfg.mu_s = hold(T[3]); cfg.mu_d = hold(T[4]); cfg.Dc = hold(T[5]); cfg.C0 = hold(T[6]);
  } catch (const std::exception &e) {
    die(e.what());
  }

  // ---- stations (io_recv_read_locate, io_funcs.cu:25-309) ------------------
  std::vector<Station> sta;
  const std::string sfile = str(par, "in_station_file");
  if (!sfile.empty()) {
    std::ifstream f(sfile);
    std::string line;
    if (!f || !next_line(f, line)) {
      std::fprintf(stderr, "cgfd_run: cannot open input station file %s\n", sfile.c_str());
    } else {
      const int n = std::atoi(line.c_str());
      for (int q = 0; q < n && next_line(f, line); q++) {
        char name[256];
        int fc = 0, fd = 0;
        float x = 0, y = 0, z = 0;
        if (std::sscanf(line.c_str(), "%255s %d %d %g %g %g", name, &fc, &fd, &x, &y, &z) != 6)
          die("station file: bad line: " + line);
        if (fc == 1) die("station file: stations by physical coordinates are not supported, give grid indices");
        Station s{ name, x - 1.0f, y - 1.0f, fd == 1 ? (float)(nk - 1) - z : z - 1.0f };
        if (s.i < 0 || s.j < 0 || s.k < 0 || (int)s.i >= ni || (int)s.j >= nj || (int)s.k >= nk) {
          std::fprintf(stderr, "cgfd_run: station %s is outside the grid, skipped\n", name);
          continue;
        }
        sta.push_back(s);
      }
    }
  }
  std::vector<FaultStation> fsta;
  const std::string ffile = str(par, "fault_station_file");
  if (!ffile.empty()) {
    std::ifstream f(ffile);
    std::string line;
    if (!f || !next_line(f, line)) {
      std::fprintf(stderr, "cgfd_run: cannot open input fault station file %s\n", ffile.c_str());
    } else {
      const int n = std::atoi(line.c_str());
      for (int q = 0; q < n && next_line(f, line); q++) {
        char name[256];
        int fid = 0;
        float y = 0, z = 0;
        if (std::sscanf(line.c_str(), "%255s %d %g %g", name, &fid, &y, &z) != 4)
          die("fault station file: bad line: " + line);
        FaultStation s{ name, fid - 1, y - 1.0f, z - 1.0f };
        if (s.fault < 0 || s.fault >= cfg.num_faults || s.j < 0 || s.k < 0 || (int)s.j >= nj || (int)s.k >= nk)
          die("fault station " + std::string(name) + " is outside the fault plane");
        fsta.push_back(s);
      }
    }
  }
  std::vector<float> sijk, fjk;
  std::vector<int> ffault;
  for (const Station &s : sta) { sijk.push_back(s.i); sijk.push_back(s.j); sijk.push_back(s.k); }
  for (const FaultStation &s : fsta) { ffault.push_back(s.fault); fjk.push_back(s.j); fjk.push_back(s.k); }
  cfg.num_stations = (int)sta.size();
  cfg.station_ijk = sijk.empty() ? nullptr : sijk.data();
  cfg.num_fault_stations = (int)fsta.size();
  cfg.fault_station_fault = ffault.empty() ? nullptr : ffault.data();
  cfg.fault_station_jk = fjk.empty() ? nullptr : fjk.data();
  cfg.max_records = nt_total;

  if (const Value *mm = par.get("metric_calculation_method"))
    if (mm->get("import")) die("metric_calculation_method: import is not supported (the metric is calculated)");
  const std::string out_dir = str(par, "output_dir", ".");

  // ---- set-up and run -----------------------------------------------------
  if (check_only) {
    cgfd_setup *su = nullptr;
    check(cgfd_prepare(&cfg, &su), "set-up");
    float dtmax = 0.f;
    check(cgfd_setup_dt_max(su, &dtmax), "set-up");
    cgfd_setup_free(su);
    std::fprintf(stdout, "grid %d x %d x %d, dt %g (max %g), %d steps, %d fault(s), dynamic_method %d, "
                 "free surface %d, %d station(s), %d fault station(s)\n", ni, nj, nk, dt, dtmax, nt_total,
                 cfg.num_faults, cfg.dynamic_method, cfg.free_surface, cfg.num_stations, cfg.num_fault_stations);
    return 0;
  }
  check(cgfd_select_device(gpu), "select GPU");
  cgfd_setup *su = nullptr;
  check(cgfd_prepare(&cfg, &su), "set-up");
  const size_t np = (size_t)ni * nj * nk;
  std::vector<float> cx(np), cy(np), cz(np);
  check(cgfd_setup_coords(su, cx.data(), cy.data(), cz.data()), "coordinates");
  cgfd_solver *s = nullptr;
  check(cgfd_upload(su, &s), "upload");
  cgfd_setup_free(su);
  auto at = [&](int i, int j, int k) { return (size_t)i + (size_t)ni * ((size_t)j + (size_t)nj * k); };

  struct FaultFile {
    cgfd_nc::Writer *w;
    int vtime, vf[CGFD_FAULT_NFIELD];
  };
  std::vector<FaultFile> ff;
  const char *fnames[CGFD_FAULT_NFIELD] = { "Tn", "Ts1", "Ts2", "Vs", "Vs1", "Vs2", "Slip", "Slip1", "Slip2",
                                           "Peak_vs", "Init_t0" };
  try {
    for (int f = 0; f < cfg.num_faults; f++) {
      const std::string file = out_dir + "/fault_i" + std::to_string(cfg.fault_x_index[f]) + "_px0_py0_pz0.nc";
      FaultFile F{ new cgfd_nc::Writer(file), 0, {} };
      const int dt_ = F.w->def_dim("time", 0), dk = F.w->def_dim("k", nk), dj = F.w->def_dim("j", nj);
      F.vtime = F.w->def_var("time", cgfd_nc::FLOAT, { dt_ });
      for (int q = 0; q < 9; q++) F.vf[q] = F.w->def_var(fnames[q], cgfd_nc::FLOAT, { dt_, dk, dj });
      for (int q = 9; q < 11; q++) F.vf[q] = F.w->def_var(fnames[q], cgfd_nc::FLOAT, { dk, dj });
      // index of the fault plane with the 3 ghost points, process grid coordinates
      F.w->put_gatt_int("i_index_with_ghosts_in_this_thread", { cfg.fault_x_index[f] - 1 + 3 });
      F.w->put_gatt_int("coords_of_mpi_topo", { 0, 0, 0 });
      F.w->end_define();
      ff.push_back(F);
    }
  } catch (const std::exception &e) {
    die(e.what());
  }

  std::vector<float> fout((size_t)CGFD_FAULT_NFIELD * nk * nj);
  // the fault records of up to kChunk output steps per call, taken while
  // the steps run into page-locked memory (cgfd_run_fault_output); a writer
  // thread puts one chunk's records into the files while the next chunk
  // steps, from the other of two buffers
  const int kChunk = 32;
  const size_t rec_floats = (size_t)cfg.num_faults * CGFD_FAULT_NFIELD * nk * nj;
  float *recs[2] = { nullptr, nullptr };
  for (int b = 0; b < 2; b++)
    check(cgfd_host_alloc(kChunk * rec_floats * sizeof(float), (void **)&recs[b]), "output buffer");
  std::string write_error;
  auto write_chunk = [&](const float *buf, int it0, int nrec) {
    try {
      for (int r = 0; r < nrec; r++) {
        const int rit = ((it0 + skip - 1) / skip + r) * skip;   // step index of record r
        const float tcur = (float)(rit * dt + t0);
        for (int f = 0; f < cfg.num_faults; f++) {
          const float *src = buf + r * rec_floats + (size_t)f * CGFD_FAULT_NFIELD * nk * nj;
          ff[f].w->put_record_float(ff[f].vtime, rit / skip, &tcur);
          for (int q = 0; q < 9; q++) ff[f].w->put_record_float(ff[f].vf[q], rit / skip, src + (size_t)q * nk * nj);
        }
      }
    } catch (const std::exception &e) {
      write_error = e.what();
    }
  };
  std::thread writer;
  int it = 0, chunk = 0;
  std::fprintf(stdout, "start time loop ...\n");
  const auto t_loop = std::chrono::steady_clock::now();
  while (it < nt_total) {
    const int n = std::min(kChunk * skip, nt_total - it);
    int nrec = 0;
    float *buf = recs[chunk & 1];          // its previous writer was joined below
    const int rc = cgfd_run_fault_output(s, n, skip, buf, kChunk, &nrec);
    if (writer.joinable()) writer.join();
    check(rc, "time steps");
    if (!write_error.empty()) die(write_error);
    writer = std::thread(write_chunk, buf, it, nrec);
    it += n;
    chunk++;
  }
  if (writer.joinable()) writer.join();
  if (!write_error.empty()) die(write_error);
  for (int b = 0; b < 2; b++) cgfd_host_free(recs[b]);
  // wall time of the time loop with its per-step fault output, the span of
  // the reference's "Runing Time" (main_curv_col_el_3d.cu:705-724)
  const double loop_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop).count();
  std::fprintf(stdout, "time loop: %.3f s for %d steps, %.3f Gpt-updates/s\n", loop_s, nt_total,
               (double)ni * nj * nk * nt_total / loop_s / 1e9);
  for (int f = 0; f < cfg.num_faults; f++) {
    check(cgfd_get_fault_all(s, f, fout.data()), "fault output");
    ff[f].w->put_float(ff[f].vf[9], fout.data() + (size_t)9 * nk * nj);
    ff[f].w->put_float(ff[f].vf[10], fout.data() + (size_t)10 * nk * nj);
    ff[f].w->close();
    delete ff[f].w;
  }

  // ---- seismograms (io_recv_output_sac and friends) -----------------------
  // the reference passes (x, y, z, dt) as station latitude, longitude,
  // elevation and depth, with zeros for the event
  int nrec = 0;
  const char *cnames[9] = { "Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Tyz", "Txz", "Txy" };
  if (!sta.empty()) {
    check(cgfd_get_stations(s, nullptr, &nrec), "stations");
    std::vector<float> seis((size_t)sta.size() * 9 * nrec);
    check(cgfd_get_stations(s, seis.data(), &nrec), "stations");
    for (size_t r = 0; r < sta.size(); r++) {
      const size_t p = at((int)sta[r].i, (int)sta[r].j, (int)sta[r].k);
      const float x = cx[p], y = cy[p], z = cz[p];
      float *tr = seis.data() + r * 9 * nrec;
      for (int c = 0; c < 9; c++)
        if (!cgfd_sac::write(out_dir + "/" + sta[r].name + "." + cnames[c] + ".sac", tr + (size_t)c * nrec, nrec,
                             (float)dt, 0, 0, 0, 0, x, y, z, (float)dt))
          die("cannot write SAC files in " + out_dir);
    }
  }
  if (!fsta.empty()) {
    int nf = 0;
    check(cgfd_get_fault_stations(s, nullptr, &nf), "fault stations");
    std::vector<float> fseis((size_t)fsta.size() * 9 * nf);
    check(cgfd_get_fault_stations(s, fseis.data(), &nf), "fault stations");
    for (size_t r = 0; r < fsta.size(); r++) {
      const size_t p = at(cfg.fault_x_index[fsta[r].fault] - 1, (int)std::floor(fsta[r].j), (int)std::floor(fsta[r].k));
      for (int c = 0; c < 9; c++)
        if (!cgfd_sac::write(out_dir + "/fault_" + fsta[r].name + "." + fnames[c] + ".sac",
                             fseis.data() + (r * 9 + c) * (size_t)nf, nf, (float)dt, 0, 0, 0, 0, cx[p], cy[p],
                             cz[p], (float)dt))
          die("cannot write SAC files in " + out_dir);
    }
  }
  if (!sta.empty()) {
    // strain at the stations from the stress traces and the medium at the
    // station's base grid point (io_recv_output_sac_el_iso_strain)
    std::vector<float> seis((size_t)sta.size() * 9 * nrec);
    check(cgfd_get_stations(s, seis.data(), &nrec), "stations");
    const char *enames[6] = { "Exx", "Eyy", "Ezz", "Eyz", "Exz", "Exy" };
    for (size_t r = 0; r < sta.size(); r++) {
      const size_t p = at((int)sta[r].i, (int)sta[r].j, (int)sta[r].k);
      const float lam = cfg.lambda[p], mu = cfg.mu[p];
      const float E1 = (float)((lam + mu) / (mu * (3.0 * lam + 2.0 * mu)));
      const float E2 = (float)(-lam / (2.0 * mu * (3.0 * lam + 2.0 * mu)));
      const float E3 = (float)(1.0 / mu);
      float *T = seis.data() + r * 9 * nrec;
      float *Txx = T + 3 * (size_t)nrec, *Tyy = T + 4 * (size_t)nrec, *Tzz = T + 5 * (size_t)nrec;
      float *Tyz = T + 6 * (size_t)nrec, *Txz = T + 7 * (size_t)nrec, *Txy = T + 8 * (size_t)nrec;
      for (int q = 0; q < nrec; q++) {
        const float E0 = E2 * (Txx[q] + Tyy[q] + Tzz[q]);
        Txx[q] = E0 - (E2 - E1) * Txx[q];
        Tyy[q] = E0 - (E2 - E1) * Tyy[q];
        Tzz[q] = E0 - (E2 - E1) * Tzz[q];
        Tyz[q] = 0.5f * E3 * Tyz[q];
        Txz[q] = 0.5f * E3 * Txz[q];
        Txy[q] = 0.5f * E3 * Txy[q];
      }
      const float x = cx[p], y = cy[p], z = cz[p];
      for (int c = 0; c < 6; c++)
        if (!cgfd_sac::write(out_dir + "/" + sta[r].name + "." + enames[c] + ".sac", T + (size_t)(3 + c) * nrec, nrec,
                             (float)dt, 0, 0, 0, 0, x, y, z, (float)dt))
          die("cannot write SAC files in " + out_dir);
    }
  }
  if (cfg.free_surface) {
    // peaks on the ghost-inclusive surface plane [ny][nx], zero in the
    // ghosts, as PG_slice_output writes them
    const int nx = ni + 6, ny = nj + 6;
    std::vector<float> pk((size_t)CGFD_NPEAK * ni * nj), plane((size_t)nx * ny);
    check(cgfd_get_surface_peaks(s, pk.data()), "surface peaks");
    const char *pnames[CGFD_NPEAK] = { "PGV", "PGVh", "PGVx", "PGVy", "PGVz", "PGA", "PGAh", "PGAx",
                                       "PGAy", "PGAz", "PGD", "PGDh", "PGDx", "PGDy", "PGDz" };
    try {
      cgfd_nc::Writer w(out_dir + "/PG_V_A_D_px0_py0_pz0.nc");
      const int dj = w.def_dim("j", ny), di = w.def_dim("i", nx);
      int vid[CGFD_NPEAK];
      for (int c = 0; c < CGFD_NPEAK; c++) vid[c] = w.def_var(pnames[c], cgfd_nc::FLOAT, { dj, di });
      w.put_gatt_int("global_index_of_first_physical_points", { 0, 0 });
      w.put_gatt_int("count_index_of_physical_points", { ni, nj });
      w.put_gatt_int("coords_of_mpi_topo", { 0, 0, 0 });
      w.end_define();
      for (int c = 0; c < CGFD_NPEAK; c++) {
        for (int j = 0; j < nj; j++)
          std::memcpy(plane.data() + (size_t)(j + 3) * nx + 3, pk.data() + ((size_t)c * nj + j) * ni, (size_t)ni * 4);
        w.put_float(vid[c], plane.data());
      }
      w.close();
    } catch (const std::exception &e) {
      die(e.what());
    }
  }
  cgfd_destroy(s);
  std::fprintf(stdout, "done: %d steps\n", nt_total);
  return 0;
}
