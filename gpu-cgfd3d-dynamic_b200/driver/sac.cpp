// sac.cpp -- SAC header layout of the published format: 70 floats, 15
// integers, 20 enumerated values, 5 logicals, then 8-byte character fields
// (the second one, the event name, is 16 bytes): 632 bytes.
#include "sac.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

namespace cgfd_sac {

namespace {
// float word indices
enum { DELTA = 0, B = 5, E = 6, STLA = 31, STLO = 32, STEL = 33, STDP = 34, EVLA = 35, EVLO = 36,
       EVEL = 37, EVDP = 38, CMPAZ = 57, CMPINC = 58 };
// integer word indices (from the start of the header)
enum { NVHDR = 76, NPTS = 79, IFTYPE = 85, LEVEN = 105 };
const float kFloatUndef = -12345.0f;
const int32_t kIntUndef = -12345;
const int kITime = 1;
}  // namespace

bool write(const std::string &path, const float *data, int npts, float delta, float evla, float evlo,
           float evel, float evdp, float stla, float stlo, float stel, float stdp) {
  float fh[70];
  int32_t ih[40];
  char kh[192];
  for (float &x : fh) x = kFloatUndef;
  for (int32_t &x : ih) x = kIntUndef;
  // 8-byte fields at 0 and 24..184, the 16-byte event name at 8 (its
  // undefined value is 8 characters and 8 NULs)
  std::memcpy(kh + 0, "-12345  ", 8);
  std::memcpy(kh + 8, "-12345  \0\0\0\0\0\0\0\0", 16);
  for (int off = 24; off < 192; off += 8) std::memcpy(kh + off, "-12345  ", 8);
  fh[DELTA] = delta; fh[B] = 0.0f; fh[E] = delta * (float)(npts - 1);
  fh[STLA] = stla; fh[STLO] = stlo; fh[STEL] = stel; fh[STDP] = stdp;
  fh[EVLA] = evla; fh[EVLO] = evlo; fh[EVEL] = evel; fh[EVDP] = evdp;
  fh[CMPAZ] = 0.0f; fh[CMPINC] = 0.0f;
  ih[NVHDR - 70] = 6; ih[NPTS - 70] = npts; ih[IFTYPE - 70] = kITime; ih[LEVEN - 70] = 1;
  // station and component names: "-12345" and two NULs
  std::memcpy(kh + 0, "-12345\0\0", 8);
  std::memcpy(kh + 160, "-12345\0\0", 8);                     // kcmpnm, the 21st field
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(fh, 4, 70, f) == 70 && std::fwrite(ih, 4, 40, f) == 40 &&
            std::fwrite(kh, 1, 192, f) == 192 &&
            std::fwrite(data, 4, (size_t)npts, f) == (size_t)npts;
  ok = std::fclose(f) == 0 && ok;
  return ok;
}

}  // namespace cgfd_sac
