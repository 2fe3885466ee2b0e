// ncclassic.h -- reader and writer of netCDF classic files.
//
// The solver's inputs (fault_coord_<id>.nc, init_stress_<id>.nc, imported
// coordinates and media) and its fault output (fault_i<x>_px0_py0_pz0.nc)
// are netCDF classic files (src/forward/gd_t.cu:548-575,
// fault_info.cu:1077-1187, io_funcs.cu:1911-2164).  This is a
// self-contained implementation of the published classic format (format
// version 1, and version 2 with 64-bit offsets for reading): big-endian
// header of dimensions, attributes and variables, fixed-size variables
// followed by records of the record variables.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace cgfd_nc {

enum Type { BYTE = 1, CHAR = 2, SHORT = 3, INT = 4, FLOAT = 5, DOUBLE = 6 };

struct Dim {
  std::string name;
  size_t len = 0;          // 0 for the record (unlimited) dimension
};

struct Att {
  std::string name;
  Type type = INT;
  std::vector<uint8_t> raw;   // values as stored (big-endian, unpadded)
  size_t nelems = 0;
};

struct Var {
  std::string name;
  std::vector<int> dims;
  std::vector<Att> atts;
  Type type = FLOAT;
  uint64_t vsize = 0, begin = 0;
  bool record = false;
};

// Read-only view of a classic file (whole header parsed at open).
class Reader {
 public:
  explicit Reader(const std::string &path);   // throws std::runtime_error
  ~Reader();
  Reader(const Reader &) = delete;
  Reader &operator=(const Reader &) = delete;
  int var(const std::string &name) const;      // -1 when absent
  const Var &var_at(int v) const { return vars_[v]; }
  size_t dim_len(int d) const { return d == rec_dim_ ? numrecs_ : dims_[d].len; }
  // hyperslab of a FLOAT or DOUBLE variable as float, C order
  void get_float(int v, const std::vector<size_t> &start, const std::vector<size_t> &count, float *out) const;
  void get_float_all(int v, float *out) const;

 private:
  FILE *f_ = nullptr;
  std::string path_;
  size_t numrecs_ = 0;
  int rec_dim_ = -1;
  uint64_t recsize_ = 0;
  std::vector<Dim> dims_;
  std::vector<Att> gatts_;
  std::vector<Var> vars_;
};

// Writer of a classic (version 1) file: define, end_define, then put.
class Writer {
 public:
  explicit Writer(const std::string &path);   // throws std::runtime_error
  ~Writer();
  Writer(const Writer &) = delete;
  Writer &operator=(const Writer &) = delete;
  int def_dim(const std::string &name, size_t len);    // len 0: record dimension
  int def_var(const std::string &name, Type type, const std::vector<int> &dims);
  void put_gatt_int(const std::string &name, const std::vector<int> &vals);
  void end_define();
  // one record of a record variable, or a whole fixed-size variable
  void put_record_float(int v, size_t rec, const float *data);
  void put_float(int v, const float *data);
  void close();

 private:
  FILE *f_ = nullptr;
  std::string path_;
  std::vector<Dim> dims_;
  std::vector<Att> gatts_;
  std::vector<Var> vars_;
  size_t numrecs_ = 0;
  uint64_t recsize_ = 0;
  bool defined_ = false;
  void write_numrecs();
};

}  // namespace cgfd_nc
