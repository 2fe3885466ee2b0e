/*
 * netcdf.h -- minimal stand-in for the netCDF C interface, test
 * infrastructure.
 *
 * The reference's own unmodified sources read their inputs
 * (fault_coord_<id>.nc, init_stress_<id>.nc, coord / media files) and write
 * their fault output (fault_i<x>_px0_py0_pz0.nc) through the netCDF library
 * (gd_t.cu:548-575,856-925; fault_info.cu:1077-1187; md_t.cu:230-288;
 * io_funcs.cu:1911-2164).  This header declares only the calls they make,
 * implemented in refshim.cpp over netCDF classic files: reads of FLOAT
 * variables (whole or hyperslab) and writes of FLOAT variables, including
 * records of the unlimited dimension, with integer global attributes.
 * A file being written is kept in memory and written out at nc_close.
 */
#ifndef CGFD_REFSHIM_NETCDF_H
#define CGFD_REFSHIM_NETCDF_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NC_NOERR         0
#define NC_EINVAL      (-36)
#define NC_ENOTVAR     (-49)
#define NC_EBADID      (-33)
#define NC_ENOTNC      (-51)
#define NC_EIO         (-68)

#define NC_NOWRITE       0x0000
#define NC_WRITE         0x0001
#define NC_CLOBBER       0x0000
#define NC_NOCLOBBER     0x0004
#define NC_64BIT_OFFSET  0x0200
#define NC_UNLIMITED     0L
#define NC_GLOBAL        (-1)

typedef int nc_type;
#define NC_BYTE   1
#define NC_CHAR   2
#define NC_SHORT  3
#define NC_INT    4
#define NC_FLOAT  5
#define NC_DOUBLE 6

const char *nc_strerror(int err);
int nc_create(const char *path, int cmode, int *ncidp);
int nc_open(const char *path, int mode, int *ncidp);
int nc_def_dim(int ncid, const char *name, size_t len, int *idp);
int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimidsp, int *varidp);
int nc_put_att_int(int ncid, int varid, const char *name, nc_type xtype, size_t len, const int *op);
int nc_enddef(int ncid);
int nc_inq_varid(int ncid, const char *name, int *varidp);
int nc_put_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, const float *op);
int nc_put_var_float(int ncid, int varid, const float *op);
int nc_put_var1_float(int ncid, int varid, const size_t *indexp, const float *op);
int nc_get_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, float *ip);
int nc_get_var(int ncid, int varid, void *ip);
int nc_close(int ncid);

#ifdef __cplusplus
}
#endif
#endif /* CGFD_REFSHIM_NETCDF_H */
