// refshim.cpp -- single-rank MPI and netCDF-classic stand-ins (mpi.h,
// netcdf.h in this directory), test infrastructure.
//
// Linked only into oracle/_ref/cgfd_ref_main, the reference's own
// unmodified sources built by oracle/build_ref.py.  The netCDF half reads
// and writes classic files through the project's classic-format reader and
// writer (gpu-cgfd3d-dynamic_b200/driver/ncclassic.cpp), which the tests
// check against scipy's independent implementation.
#include "mpi.h"
#include "netcdf.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ncclassic.h"

// ---------------------------------------------------------------- MPI -----
extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) {
  std::fprintf(stderr, "MPI_Abort(%d)\n", code);
  std::fflush(stderr);
  std::exit(code == 0 ? 1 : code);
}
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  if (sendbuf != recvbuf) std::memmove(recvbuf, sendbuf, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int, MPI_Datatype,
                  MPI_Comm) {
  if (sendbuf != recvbuf) std::memmove(recvbuf, sendbuf, (size_t)scount * (size_t)stype);
  return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm comm, int, const int dims[], const int[], int, MPI_Comm *cart) {
  // mympi_set (mympi_t.cu:32) builds a 3-D topology from the par file's
  // process counts; one rank can only stand for a 1 x 1 x 1 grid
  for (int d = 0; d < 3; d++)
    if (dims[d] != 1) {
      std::fprintf(stderr, "single-rank MPI stand-in: process grid must be 1 x 1 x 1\n");
      std::exit(9);
    }
  *cart = comm;
  return MPI_SUCCESS;
}
int MPI_Cart_coords(MPI_Comm, int, int maxdims, int coords[]) {
  for (int d = 0; d < maxdims; d++) coords[d] = 0;
  return MPI_SUCCESS;
}
int MPI_Cart_shift(MPI_Comm, int, int, int *source, int *dest) {
  *source = MPI_PROC_NULL;
  *dest = MPI_PROC_NULL;
  return MPI_SUCCESS;
}
int MPI_Type_vector(int, int, int, MPI_Datatype old, MPI_Datatype *newtype) { *newtype = old; return MPI_SUCCESS; }
int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }

static void need_null(int partner, const char *what) {
  if (partner != MPI_PROC_NULL) {
    std::fprintf(stderr, "single-rank MPI stand-in: %s with partner %d\n", what, partner);
    std::exit(9);
  }
}
int MPI_Send_init(const void *, int, MPI_Datatype, int dest, int, MPI_Comm, MPI_Request *req) {
  need_null(dest, "MPI_Send_init");
  *req = 0;
  return MPI_SUCCESS;
}
int MPI_Recv_init(void *, int, MPI_Datatype, int source, int, MPI_Comm, MPI_Request *req) {
  need_null(source, "MPI_Recv_init");
  *req = 0;
  return MPI_SUCCESS;
}
int MPI_Startall(int, MPI_Request[]) { return MPI_SUCCESS; }
int MPI_Waitall(int, MPI_Request[], MPI_Status *) { return MPI_SUCCESS; }
int MPI_Sendrecv(const void *, int, MPI_Datatype, int dest, int, void *, int, MPI_Datatype, int source, int,
                 MPI_Comm, MPI_Status *) {
  need_null(dest, "MPI_Sendrecv");
  need_null(source, "MPI_Sendrecv");
  return MPI_SUCCESS;
}

}  // extern "C"

// ------------------------------------------------------------- netCDF -----
namespace {

struct DefVar {
  std::string name;
  std::vector<int> dims;
};

struct File {
  std::unique_ptr<cgfd_nc::Reader> r;   // open for reading
  std::unique_ptr<cgfd_nc::Writer> w;   // created for writing
  std::vector<size_t> dim_len;          // of a file being written (0: record)
  std::vector<DefVar> vars;
};

std::map<int, File> g_files;
int g_next = 1;
std::string g_msg;

File *get(int ncid) {
  auto f = g_files.find(ncid);
  return f == g_files.end() ? nullptr : &f->second;
}

// elements of one record (record variable) or of the whole variable
size_t var_elems(const File &F, int v, bool *record) {
  const DefVar &d = F.vars[v];
  *record = !d.dims.empty() && F.dim_len[d.dims[0]] == 0;
  size_t n = 1;
  for (size_t q = *record ? 1 : 0; q < d.dims.size(); q++) n *= F.dim_len[d.dims[q]];
  return n;
}

int err(int code, const std::string &m) {
  g_msg = m;
  return code;
}

}  // namespace

extern "C" {

const char *nc_strerror(int e) {
  static std::string s;
  s = "netCDF stand-in error " + std::to_string(e) + (g_msg.empty() ? "" : ": " + g_msg);
  return s.c_str();
}

int nc_create(const char *path, int, int *ncidp) {
  try {
    File F;
    F.w.reset(new cgfd_nc::Writer(path));
    const int id = g_next++;
    g_files[id] = std::move(F);
    *ncidp = id;
    return NC_NOERR;
  } catch (const std::exception &e) {
    return err(NC_EIO, e.what());
  }
}

int nc_open(const char *path, int, int *ncidp) {
  try {
    File F;
    F.r.reset(new cgfd_nc::Reader(path));
    const int id = g_next++;
    g_files[id] = std::move(F);
    *ncidp = id;
    return NC_NOERR;
  } catch (const std::exception &e) {
    return err(NC_ENOTNC, e.what());
  }
}

int nc_def_dim(int ncid, const char *name, size_t len, int *idp) {
  File *F = get(ncid);
  if (!F || !F->w) return err(NC_EBADID, "def_dim");
  *idp = F->w->def_dim(name, len);
  F->dim_len.push_back(len);
  return NC_NOERR;
}

int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimidsp, int *varidp) {
  File *F = get(ncid);
  if (!F || !F->w) return err(NC_EBADID, "def_var");
  if (xtype != NC_FLOAT) return err(NC_EINVAL, std::string("only FLOAT variables: ") + name);
  std::vector<int> d(dimidsp, dimidsp + ndims);
  *varidp = F->w->def_var(name, cgfd_nc::FLOAT, d);
  F->vars.push_back({ name, d });
  return NC_NOERR;
}

int nc_put_att_int(int ncid, int varid, const char *name, nc_type, size_t len, const int *op) {
  File *F = get(ncid);
  if (!F || !F->w) return err(NC_EBADID, "put_att_int");
  if (varid != NC_GLOBAL) return err(NC_EINVAL, "only global attributes");
  F->w->put_gatt_int(name, std::vector<int>(op, op + len));
  return NC_NOERR;
}

int nc_enddef(int ncid) {
  File *F = get(ncid);
  if (!F || !F->w) return err(NC_EBADID, "enddef");
  try {
    F->w->end_define();
  } catch (const std::exception &e) {
    return err(NC_EIO, e.what());
  }
  return NC_NOERR;
}

int nc_inq_varid(int ncid, const char *name, int *varidp) {
  File *F = get(ncid);
  if (!F) return err(NC_EBADID, "inq_varid");
  if (F->r) {
    const int v = F->r->var(name);
    if (v < 0) return err(NC_ENOTVAR, name);
    *varidp = v;
    return NC_NOERR;
  }
  for (size_t v = 0; v < F->vars.size(); v++)
    if (F->vars[v].name == name) { *varidp = (int)v; return NC_NOERR; }
  return err(NC_ENOTVAR, name);
}

// writes of whole records or whole variables, the only ones the reference
// makes (io_funcs.cu:1911-2164)
int nc_put_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, const float *op) {
  File *F = get(ncid);
  if (!F || !F->w || varid < 0 || varid >= (int)F->vars.size()) return err(NC_EBADID, "put_vara_float");
  bool record = false;
  var_elems(*F, varid, &record);
  const DefVar &d = F->vars[varid];
  for (size_t q = record ? 1 : 0; q < d.dims.size(); q++)
    if (startp[q] != 0 || countp[q] != F->dim_len[d.dims[q]])
      return err(NC_EINVAL, "partial hyperslab write of " + d.name);
  try {
    if (record) {
      if (countp[0] != 1) return err(NC_EINVAL, "one record per write: " + d.name);
      F->w->put_record_float(varid, startp[0], op);
    } else {
      F->w->put_float(varid, op);
    }
  } catch (const std::exception &e) {
    return err(NC_EIO, e.what());
  }
  return NC_NOERR;
}

int nc_put_var_float(int ncid, int varid, const float *op) {
  File *F = get(ncid);
  if (!F || !F->w || varid < 0 || varid >= (int)F->vars.size()) return err(NC_EBADID, "put_var_float");
  bool record = false;
  var_elems(*F, varid, &record);
  if (record) return err(NC_EINVAL, "put_var of a record variable");
  try {
    F->w->put_float(varid, op);
  } catch (const std::exception &e) {
    return err(NC_EIO, e.what());
  }
  return NC_NOERR;
}

int nc_put_var1_float(int ncid, int varid, const size_t *indexp, const float *op) {
  File *F = get(ncid);
  if (!F || !F->w || varid < 0 || varid >= (int)F->vars.size()) return err(NC_EBADID, "put_var1_float");
  bool record = false;
  const size_t n = var_elems(*F, varid, &record);
  if (!record || n != 1) return err(NC_EINVAL, "put_var1 only for 1-D record variables");
  try {
    F->w->put_record_float(varid, indexp[0], op);
  } catch (const std::exception &e) {
    return err(NC_EIO, e.what());
  }
  return NC_NOERR;
}

int nc_get_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, float *ip) {
  File *F = get(ncid);
  if (!F || !F->r) return err(NC_EBADID, "get_vara_float");
  try {
    const size_t nd = F->r->var_at(varid).dims.size();
    F->r->get_float(varid, std::vector<size_t>(startp, startp + nd), std::vector<size_t>(countp, countp + nd), ip);
  } catch (const std::exception &e) {
    return err(NC_EINVAL, e.what());
  }
  return NC_NOERR;
}

// whole-variable read; the reference calls it on FLOAT variables only
// (md_t.cu:265, gd_t.cu:1049)
int nc_get_var(int ncid, int varid, void *ip) {
  File *F = get(ncid);
  if (!F || !F->r) return err(NC_EBADID, "get_var");
  try {
    F->r->get_float_all(varid, static_cast<float *>(ip));
  } catch (const std::exception &e) {
    return err(NC_EINVAL, e.what());
  }
  return NC_NOERR;
}

int nc_close(int ncid) {
  File *F = get(ncid);
  if (!F) return err(NC_EBADID, "close");
  try {
    if (F->w) F->w->close();
  } catch (const std::exception &e) {
    g_files.erase(ncid);
    return err(NC_EIO, e.what());
  }
  g_files.erase(ncid);
  return NC_NOERR;
}

}  // extern "C"
