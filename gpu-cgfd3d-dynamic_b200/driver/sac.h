// sac.h -- SAC binary seismogram files (version 6 header, native byte
// order), as the solver's station output (src/lib/sacLib.cu:8-377,
// io_funcs.cu:578-617).
#pragma once
#include <string>

namespace cgfd_sac {

// One evenly sampled trace.  Header fields that the reference's writer
// sets: delta, b = 0, e = delta (npts - 1), nvhdr 6, npts, iftype ITIME,
// leven, the event and station positions, cmpaz = cmpinc = 0; kstnm and
// kcmpnm are "-12345"; every other field holds the undefined value.
// Returns false when the file cannot be written.
bool write(const std::string &path, const float *data, int npts, float delta, float evla, float evlo,
           float evel, float evdp, float stla, float stlo, float stel, float stdp);

}  // namespace cgfd_sac
