// Test helper for tests/test_driver.py: exercises the driver's netCDF
// classic reader / writer and SAC writer from the command line.
//   read FILE VAR          print every value of VAR (float), one per line
//   write FILE             write a small file shaped like the fault output
//   sac FILE               write a 5-sample SAC trace
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../gpu-cgfd3d-dynamic_b200/driver/ncclassic.h"
#include "../gpu-cgfd3d-dynamic_b200/driver/sac.h"

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const std::string mode = argv[1], path = argv[2];
  try {
    if (mode == "read" && argc > 3) {
      cgfd_nc::Reader r(path);
      const int v = r.var(argv[3]);
      if (v < 0) return 3;
      size_t n = 1;
      for (int d : r.var_at(v).dims) n *= r.dim_len(d);
      std::vector<float> out(n);
      r.get_float_all(v, out.data());
      for (float x : out) std::printf("%.9g\n", x);
      // a sub-slab of a rank-2 variable: rows 1.., columns 1..2
      if (r.var_at(v).dims.size() == 2 && r.dim_len(r.var_at(v).dims[0]) > 1 && r.dim_len(r.var_at(v).dims[1]) > 2) {
        std::vector<float> s(2 * (r.dim_len(r.var_at(v).dims[0]) - 1));
        r.get_float(v, { 1, 1 }, { r.dim_len(r.var_at(v).dims[0]) - 1, 2 }, s.data());
        std::printf("slab\n");
        for (float x : s) std::printf("%.9g\n", x);
      }
      return 0;
    }
    if (mode == "write") {
      cgfd_nc::Writer w(path);
      const int t = w.def_dim("time", 0), k = w.def_dim("k", 3), j = w.def_dim("j", 4);
      const int vt = w.def_var("time", cgfd_nc::FLOAT, { t });
      const int va = w.def_var("Tn", cgfd_nc::FLOAT, { t, k, j });
      const int vb = w.def_var("Vs", cgfd_nc::FLOAT, { t, k, j });
      const int vp = w.def_var("Peak_vs", cgfd_nc::FLOAT, { k, j });
      w.put_gatt_int("i_index_with_ghosts_in_this_thread", { 53 });
      w.put_gatt_int("coords_of_mpi_topo", { 0, 0, 0 });
      w.end_define();
      float a[12], b[12], p[12];
      for (int rec = 0; rec < 2; rec++) {
        const float tm = 0.5f * rec;
        for (int q = 0; q < 12; q++) { a[q] = 100.0f * rec + q; b[q] = -1.0f * q - rec; }
        w.put_record_float(vt, rec, &tm);
        w.put_record_float(va, rec, a);
        w.put_record_float(vb, rec, b);
      }
      for (int q = 0; q < 12; q++) p[q] = 0.25f * q;
      w.put_float(vp, p);
      w.close();
      return 0;
    }
    if (mode == "sac") {
      const float d[5] = { 1, 2, 3, 4, 5 };
      return cgfd_sac::write(path, d, 5, 0.01f, 0, 0, 0, 0, 1.5f, 2.5f, -3.5f, 0.01f) ? 0 : 4;
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 5;
  }
  return 2;
}
