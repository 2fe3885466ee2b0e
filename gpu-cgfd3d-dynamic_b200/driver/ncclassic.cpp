// ncclassic.cpp -- netCDF classic format: header parsing and writing,
// hyperslab reads of float/double variables, record writes.
#include "ncclassic.h"

#include <cstring>
#include <stdexcept>

namespace cgfd_nc {

namespace {

const uint32_t kDimTag = 0x0A, kVarTag = 0x0B, kAttTag = 0x0C;

size_t type_size(Type t) {
  switch (t) {
    case BYTE: case CHAR: return 1;
    case SHORT: return 2;
    case INT: case FLOAT: return 4;
    case DOUBLE: return 8;
  }
  return 0;
}
size_t pad4(size_t n) { return (n + 3) & ~(size_t)3; }

uint32_t be32(const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }
uint64_t be64(const uint8_t *p) { return (uint64_t)be32(p) << 32 | be32(p + 4); }
void put32(std::vector<uint8_t> &b, uint32_t v) {
  for (int s = 24; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
}
void put_name(std::vector<uint8_t> &b, const std::string &n) {
  put32(b, (uint32_t)n.size());
  b.insert(b.end(), n.begin(), n.end());
  while (b.size() % 4) b.push_back(0);
}

// cursor over the header bytes
struct Cur {
  const std::vector<uint8_t> &b;
  size_t p = 0;
  const std::string &path;
  void need(size_t n) {
    if (p + n > b.size()) throw std::runtime_error(path + ": truncated netCDF header");
  }
  uint32_t u32() { need(4); uint32_t v = be32(&b[p]); p += 4; return v; }
  uint64_t u64() { need(8); uint64_t v = be64(&b[p]); p += 8; return v; }
  std::string name() {
    const uint32_t n = u32();
    need(pad4(n));
    std::string s(reinterpret_cast<const char *>(&b[p]), n);
    p += pad4(n);
    return s;
  }
};

std::vector<Att> read_atts(Cur &c) {
  std::vector<Att> out;
  const uint32_t tag = c.u32(), n = c.u32();
  if (tag == 0 && n == 0) return out;
  if (tag != kAttTag) throw std::runtime_error(c.path + ": bad attribute list");
  for (uint32_t q = 0; q < n; q++) {
    Att a;
    a.name = c.name();
    a.type = (Type)c.u32();
    a.nelems = c.u32();
    const size_t nb = a.nelems * type_size(a.type);
    c.need(pad4(nb));
    a.raw.assign(c.b.begin() + c.p, c.b.begin() + c.p + nb);
    c.p += pad4(nb);
    out.push_back(a);
  }
  return out;
}

float to_float(Type t, const uint8_t *p) {
  if (t == FLOAT) { uint32_t u = be32(p); float f; std::memcpy(&f, &u, 4); return f; }
  uint64_t u = be64(p);
  double d;
  std::memcpy(&d, &u, 8);
  return (float)d;
}

}  // namespace

// ---------------------------------------------------------------------------
Reader::Reader(const std::string &path) : path_(path) {
  f_ = std::fopen(path.c_str(), "rb");
  if (!f_) throw std::runtime_error("cannot open " + path);
  // the header is at the front; read a generous prefix, grow if needed
  std::vector<uint8_t> b;
  size_t want = 1 << 16;
  for (;;) {
    b.resize(want);
    std::fseek(f_, 0, SEEK_SET);
    b.resize(std::fread(b.data(), 1, want, f_));
    try {
      Cur c{ b, 0, path_ };
      c.need(4);
      if (b[0] != 'C' || b[1] != 'D' || b[2] != 'F' || (b[3] != 1 && b[3] != 2))
        throw std::runtime_error(path + ": not a netCDF classic file");
      const bool off64 = b[3] == 2;
      c.p = 4;
      numrecs_ = c.u32();
      uint32_t tag = c.u32(), n = c.u32();
      if (!(tag == 0 && n == 0)) {
        if (tag != kDimTag) throw std::runtime_error(path + ": bad dimension list");
        for (uint32_t q = 0; q < n; q++) {
          Dim d;
          d.name = c.name();
          d.len = c.u32();
          if (d.len == 0) rec_dim_ = (int)q;
          dims_.push_back(d);
        }
      }
      gatts_ = read_atts(c);
      tag = c.u32(); n = c.u32();
      if (!(tag == 0 && n == 0)) {
        if (tag != kVarTag) throw std::runtime_error(path + ": bad variable list");
        for (uint32_t q = 0; q < n; q++) {
          Var v;
          v.name = c.name();
          const uint32_t nd = c.u32();
          for (uint32_t d = 0; d < nd; d++) v.dims.push_back((int)c.u32());
          v.atts = read_atts(c);
          v.type = (Type)c.u32();
          v.vsize = c.u32();
          v.begin = off64 ? c.u64() : c.u32();
          v.record = !v.dims.empty() && v.dims[0] == rec_dim_;
          vars_.push_back(v);
        }
      }
      break;
    } catch (const std::runtime_error &e) {
      if (b.size() < want || want > (1u << 28)) throw;   // whole file read: a real error
      want *= 4;
      dims_.clear(); gatts_.clear(); vars_.clear(); rec_dim_ = -1;
    }
  }
  int nrv = 0;
  for (const Var &v : vars_) if (v.record) { recsize_ += v.vsize; nrv++; }
  // a single record variable is not padded
  if (nrv == 1)
    for (const Var &v : vars_)
      if (v.record) {
        size_t e = type_size(v.type);
        for (size_t d = 1; d < v.dims.size(); d++) e *= dims_[v.dims[d]].len;
        recsize_ = e;
      }
}

Reader::~Reader() { if (f_) std::fclose(f_); }

int Reader::var(const std::string &name) const {
  for (size_t q = 0; q < vars_.size(); q++) if (vars_[q].name == name) return (int)q;
  return -1;
}

void Reader::get_float(int vi, const std::vector<size_t> &start, const std::vector<size_t> &count, float *out) const {
  const Var &v = vars_.at(vi);
  if (v.type != FLOAT && v.type != DOUBLE) throw std::runtime_error(path_ + ": " + v.name + " is not float/double");
  const size_t nd = v.dims.size();
  if (start.size() != nd || count.size() != nd) throw std::runtime_error(path_ + ": " + v.name + ": rank mismatch");
  std::vector<size_t> len(nd);
  for (size_t d = 0; d < nd; d++) {
    len[d] = dim_len(v.dims[d]);
    if (start[d] + count[d] > len[d]) throw std::runtime_error(path_ + ": " + v.name + ": slab outside the variable");
  }
  const size_t es = type_size(v.type);
  // the innermost dimension is read as one run per outer index, unless it
  // is the record dimension itself (one value per record)
  const bool rec_only = v.record && nd == 1;
  const size_t inner = rec_only ? 1 : (nd ? count[nd - 1] : 1);
  size_t nouter = rec_only ? count[0] : 1;
  for (size_t d = 0; d + 1 < nd; d++) nouter *= count[d];
  std::vector<uint8_t> run(inner * es);
  std::vector<size_t> idx(nd, 0);
  size_t o = 0;
  for (size_t q = 0; q < nouter; q++) {
    // element offset of (start + idx) within one record / the variable
    uint64_t off = v.begin;
    size_t stride = es;
    for (size_t d = nd; d-- > (v.record ? 1 : 0);) {
      off += (uint64_t)(start[d] + (d + 1 == nd ? 0 : idx[d])) * stride;
      stride *= len[d];
    }
    if (v.record) off += (uint64_t)(start[0] + (rec_only ? q : idx[0])) * recsize_;
    if (std::fseek(f_, (long)off, SEEK_SET) != 0 || std::fread(run.data(), 1, run.size(), f_) != run.size())
      throw std::runtime_error(path_ + ": short read of " + v.name);
    for (size_t e = 0; e < inner; e++) out[o++] = to_float(v.type, &run[e * es]);
    for (size_t d = nd < 2 ? 0 : nd - 1; d-- > 0;) {   // advance the outer multi-index
      if (++idx[d] < count[d]) break;
      idx[d] = 0;
    }
  }
}

void Reader::get_float_all(int vi, float *out) const {
  const Var &v = vars_.at(vi);
  std::vector<size_t> start(v.dims.size(), 0), count(v.dims.size());
  for (size_t d = 0; d < v.dims.size(); d++) count[d] = dim_len(v.dims[d]);
  get_float(vi, start, count, out);
}

// ---------------------------------------------------------------------------
Writer::Writer(const std::string &path) : path_(path) {
  f_ = std::fopen(path.c_str(), "wb+");
  if (!f_) throw std::runtime_error("cannot create " + path);
}

Writer::~Writer() { close(); }

int Writer::def_dim(const std::string &name, size_t len) {
  dims_.push_back({ name, len });
  return (int)dims_.size() - 1;
}

int Writer::def_var(const std::string &name, Type type, const std::vector<int> &dims) {
  Var v;
  v.name = name;
  v.type = type;
  v.dims = dims;
  v.record = !dims.empty() && dims_[dims[0]].len == 0;
  vars_.push_back(v);
  return (int)vars_.size() - 1;
}

void Writer::put_gatt_int(const std::string &name, const std::vector<int> &vals) {
  Att a;
  a.name = name;
  a.type = INT;
  a.nelems = vals.size();
  for (int x : vals) put32(a.raw, (uint32_t)x);
  gatts_.push_back(a);
}

void Writer::end_define() {
  // sizes: vsize is the padded size of one record (record variables) or of
  // the whole variable; fixed-size data follows the header in definition
  // order, then the records
  int nrv = 0;
  for (Var &v : vars_) {
    size_t n = type_size(v.type);
    for (size_t d = v.record ? 1 : 0; d < v.dims.size(); d++) n *= dims_[v.dims[d]].len;
    v.vsize = pad4(n);
    if (v.record) nrv++;
  }
  auto header = [&](void) {
    std::vector<uint8_t> b = { 'C', 'D', 'F', 1 };
    put32(b, (uint32_t)numrecs_);
    if (dims_.empty()) { put32(b, 0); put32(b, 0); }
    else {
      put32(b, kDimTag); put32(b, (uint32_t)dims_.size());
      for (const Dim &d : dims_) { put_name(b, d.name); put32(b, (uint32_t)d.len); }
    }
    auto atts = [&](const std::vector<Att> &as) {
      if (as.empty()) { put32(b, 0); put32(b, 0); return; }
      put32(b, kAttTag); put32(b, (uint32_t)as.size());
      for (const Att &a : as) {
        put_name(b, a.name); put32(b, a.type); put32(b, (uint32_t)a.nelems);
        b.insert(b.end(), a.raw.begin(), a.raw.end());
        while (b.size() % 4) b.push_back(0);
      }
    };
    atts(gatts_);
    if (vars_.empty()) { put32(b, 0); put32(b, 0); }
    else {
      put32(b, kVarTag); put32(b, (uint32_t)vars_.size());
      for (const Var &v : vars_) {
        put_name(b, v.name); put32(b, (uint32_t)v.dims.size());
        for (int d : v.dims) put32(b, (uint32_t)d);
        atts(v.atts);
        put32(b, v.type); put32(b, (uint32_t)v.vsize); put32(b, (uint32_t)v.begin);
      }
    }
    return b;
  };
  const size_t hsize = header().size();   // begins do not change the size
  uint64_t off = hsize;
  for (Var &v : vars_) if (!v.record) { v.begin = off; off += v.vsize; }
  recsize_ = 0;
  for (Var &v : vars_) if (v.record) { v.begin = off + recsize_; recsize_ += v.vsize; }
  if (nrv == 1)
    for (Var &v : vars_)
      if (v.record) {
        size_t n = type_size(v.type);
        for (size_t d = 1; d < v.dims.size(); d++) n *= dims_[v.dims[d]].len;
        recsize_ = n;
      }
  const std::vector<uint8_t> h = header();
  if (std::fwrite(h.data(), 1, h.size(), f_) != h.size()) throw std::runtime_error(path_ + ": write failed");
  // fixed-size variables start filled with zeros until written
  std::vector<uint8_t> zero(off - hsize, 0);
  if (!zero.empty() && std::fwrite(zero.data(), 1, zero.size(), f_) != zero.size())
    throw std::runtime_error(path_ + ": write failed");
  defined_ = true;
}

void Writer::put_record_float(int vi, size_t rec, const float *data) {
  const Var &v = vars_.at(vi);
  if (!defined_ || !v.record || v.type != FLOAT) throw std::runtime_error(path_ + ": bad record write");
  size_t n = 1;
  for (size_t d = 1; d < v.dims.size(); d++) n *= dims_[v.dims[d]].len;
  std::vector<uint8_t> b;
  b.reserve(v.vsize);
  for (size_t q = 0; q < n; q++) { uint32_t u; std::memcpy(&u, data + q, 4); put32(b, u); }
  b.resize(v.vsize, 0);
  const uint64_t off = v.begin + rec * recsize_;
  if (std::fseek(f_, (long)off, SEEK_SET) != 0 || std::fwrite(b.data(), 1, b.size(), f_) != b.size())
    throw std::runtime_error(path_ + ": write failed");
  if (rec + 1 > numrecs_) {
    // the records in between hold zeros until written
    numrecs_ = rec + 1;
    write_numrecs();
  }
}

void Writer::put_float(int vi, const float *data) {
  const Var &v = vars_.at(vi);
  if (!defined_ || v.record || v.type != FLOAT) throw std::runtime_error(path_ + ": bad variable write");
  std::vector<uint8_t> b;
  const size_t n = (v.vsize) / 4;
  size_t nv = 1;
  for (int d : v.dims) nv *= dims_[d].len;
  for (size_t q = 0; q < n; q++) {
    uint32_t u = 0;
    if (q < nv) std::memcpy(&u, data + q, 4);
    put32(b, u);
  }
  if (std::fseek(f_, (long)v.begin, SEEK_SET) != 0 || std::fwrite(b.data(), 1, b.size(), f_) != b.size())
    throw std::runtime_error(path_ + ": write failed");
}

void Writer::write_numrecs() {
  std::vector<uint8_t> b;
  put32(b, (uint32_t)numrecs_);
  std::fseek(f_, 4, SEEK_SET);
  std::fwrite(b.data(), 1, 4, f_);
}

void Writer::close() {
  if (f_) {
    if (defined_) write_numrecs();
    std::fclose(f_);
    f_ = nullptr;
  }
}

}  // namespace cgfd_nc
