// ncclassic.cpp -- NetCDF classic (CDF-1/CDF-2) I/O from the format specification:
//   header  = 'C' 'D' 'F' version, numrecs, dim_list, gatt_list, var_list
//   lists   = ABSENT (two zero words) | tag nelems items; tags 0x0A dims, 0x0C atts, 0x0B vars
//   names   = nelems + bytes padded to 4; attribute values padded to 4
//   var     = name, ndims, dimids, vatt_list, nc_type, vsize, begin (32-bit in CDF-1, 64 in CDF-2)
// Everything is big-endian. Record variables interleave per record (recsize = sum of vsizes).
#include "ncclassic.h"

#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace cgfd {
namespace nc {

namespace {

constexpr uint32_t TAG_DIM = 0x0A, TAG_VAR = 0x0B, TAG_ATT = 0x0C;

int type_size(int t) {
  switch (t) {
    case BYTE: case CHAR: return 1;
    case SHORT: return 2;
    case INT: case FLOAT: return 4;
    case DOUBLE: return 8;
  }
  throw std::runtime_error("netcdf: unknown nc_type " + std::to_string(t));
}

uint64_t pad4(uint64_t n) { return (n + 3) & ~uint64_t(3); }

struct Reader {
  std::vector<unsigned char> buf;
  size_t p = 0;
  uint32_t u32() {
    if (p + 4 > buf.size()) throw std::runtime_error("netcdf: truncated header");
    uint32_t v = (uint32_t)buf[p] << 24 | (uint32_t)buf[p + 1] << 16 | (uint32_t)buf[p + 2] << 8 | buf[p + 3];
    p += 4;
    return v;
  }
  uint64_t u64() {
    uint64_t hi = u32();
    return hi << 32 | u32();
  }
  std::string name() {
    uint32_t n = u32();
    if (p + n > buf.size()) throw std::runtime_error("netcdf: truncated name");
    std::string s((const char *)&buf[p], n);
    p += pad4(n);
    return s;
  }
};

double be_value(const unsigned char *q, int t) {
  switch (t) {
    case BYTE: return (double)(int8_t)q[0];
    case SHORT: return (double)(int16_t)((q[0] << 8) | q[1]);
    case INT: {
      uint32_t v = (uint32_t)q[0] << 24 | (uint32_t)q[1] << 16 | (uint32_t)q[2] << 8 | q[3];
      return (double)(int32_t)v;
    }
    case FLOAT: {
      uint32_t v = (uint32_t)q[0] << 24 | (uint32_t)q[1] << 16 | (uint32_t)q[2] << 8 | q[3];
      float f;
      memcpy(&f, &v, 4);
      return f;
    }
    case DOUBLE: {
      uint64_t v = 0;
      for (int n = 0; n < 8; n++) v = v << 8 | q[n];
      double d;
      memcpy(&d, &v, 8);
      return d;
    }
  }
  return 0.0;
}

std::vector<Att> read_atts(Reader &r) {
  std::vector<Att> out;
  uint32_t tag = r.u32(), n = r.u32();
  if (tag == 0 && n == 0) return out;
  if (tag != TAG_ATT) throw std::runtime_error("netcdf: bad attribute list");
  for (uint32_t a = 0; a < n; a++) {
    Att at;
    at.name = r.name();
    at.type = (int)r.u32();
    uint32_t ne = r.u32();
    int ts = type_size(at.type);
    if (r.p + (size_t)ne * ts > r.buf.size()) throw std::runtime_error("netcdf: truncated attribute");
    if (at.type == CHAR) at.text.assign((const char *)&r.buf[r.p], ne);
    else
      for (uint32_t e = 0; e < ne; e++) at.num.push_back(be_value(&r.buf[r.p + (size_t)e * ts], at.type));
    r.p += pad4((uint64_t)ne * ts);
    out.push_back(at);
  }
  return out;
}

struct Writer {
  std::vector<unsigned char> b;
  void u32(uint32_t v) {
    unsigned char q[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8), (unsigned char)v};
    b.insert(b.end(), q, q + 4);
  }
  void u64(uint64_t v) { u32((uint32_t)(v >> 32)); u32((uint32_t)v); }
  void name(const std::string &s) {
    u32((uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    while (b.size() % 4) b.push_back(0);
  }
};

void put_atts(Writer &w, const std::vector<Att> &atts) {
  if (atts.empty()) { w.u32(0); w.u32(0); return; }
  w.u32(TAG_ATT);
  w.u32((uint32_t)atts.size());
  for (const Att &a : atts) {
    w.name(a.name);
    w.u32((uint32_t)a.type);
    if (a.type == CHAR) {
      w.u32((uint32_t)a.text.size());
      w.b.insert(w.b.end(), a.text.begin(), a.text.end());
    } else if (a.type == INT) {
      w.u32((uint32_t)a.num.size());
      for (double v : a.num) w.u32((uint32_t)(int32_t)v);
    } else if (a.type == FLOAT) {
      w.u32((uint32_t)a.num.size());
      for (double v : a.num) { float f = (float)v; uint32_t u; memcpy(&u, &f, 4); w.u32(u); }
    } else if (a.type == DOUBLE) {
      w.u32((uint32_t)a.num.size());
      for (double v : a.num) { uint64_t u; memcpy(&u, &v, 8); w.u64(u); }
    } else {
      throw std::runtime_error("netcdf: unsupported attribute type for writing");
    }
    while (w.b.size() % 4) w.b.push_back(0);
  }
}

}  // namespace

int File::find_var(const std::string &name) const {
  for (size_t v = 0; v < vars.size(); v++)
    if (vars[v].name == name) return (int)v;
  return -1;
}

const Att *File::find_gatt(const std::string &name) const {
  for (const Att &a : gatts)
    if (a.name == name) return &a;
  return nullptr;
}

std::vector<uint64_t> File::shape(int varid) const {
  std::vector<uint64_t> s;
  for (int d : vars[varid].dimids) s.push_back(dims[d].len == 0 ? numrecs : dims[d].len);
  return s;
}

File read_header(const std::string &path) {
  FILE *fp = fopen(path.c_str(), "rb");
  if (!fp) throw std::runtime_error("cannot open " + path);
  Reader r;
  // the header is small; read up to 1 MiB (grows if needed)
  size_t want = 1 << 20;
  r.buf.resize(want);
  size_t got = fread(r.buf.data(), 1, want, fp);
  fclose(fp);
  r.buf.resize(got);
  if (got < 8 || memcmp(r.buf.data(), "CDF", 3) != 0) throw std::runtime_error(path + ": not a NetCDF classic file");
  File f;
  f.version = r.buf[3];
  if (f.version != 1 && f.version != 2) throw std::runtime_error(path + ": unsupported NetCDF version");
  r.p = 4;
  f.numrecs = r.u32();
  uint32_t tag = r.u32(), n = r.u32();
  if (!(tag == 0 && n == 0)) {
    if (tag != TAG_DIM) throw std::runtime_error("netcdf: bad dim list");
    for (uint32_t d = 0; d < n; d++) {
      Dim dm;
      dm.name = r.name();
      dm.len = r.u32();
      f.dims.push_back(dm);
    }
  }
  f.gatts = read_atts(r);
  tag = r.u32();
  n = r.u32();
  if (!(tag == 0 && n == 0)) {
    if (tag != TAG_VAR) throw std::runtime_error("netcdf: bad var list");
    for (uint32_t v = 0; v < n; v++) {
      Var var;
      var.name = r.name();
      uint32_t nd = r.u32();
      for (uint32_t d = 0; d < nd; d++) var.dimids.push_back((int)r.u32());
      var.atts = read_atts(r);
      var.type = (int)r.u32();
      var.vsize = r.u32();
      var.begin = f.version == 1 ? r.u32() : r.u64();
      f.vars.push_back(var);
    }
  }
  return f;
}

std::vector<float> read_var(const std::string &path, const File &f, const std::string &name) {
  int vid = f.find_var(name);
  if (vid < 0) throw std::runtime_error(path + ": no variable '" + name + "'");
  const Var &v = f.vars[vid];
  std::vector<uint64_t> shp = f.shape(vid);
  uint64_t n = 1;
  for (uint64_t s : shp) n *= s;
  int ts = type_size(v.type);
  std::vector<float> out(n);
  FILE *fp = fopen(path.c_str(), "rb");
  if (!fp) throw std::runtime_error("cannot open " + path);
  bool is_rec = !v.dimids.empty() && f.dims[v.dimids[0]].len == 0;
  std::vector<unsigned char> tmp;
  auto read_at = [&](uint64_t off, uint64_t cnt, float *dst) {
    tmp.resize(cnt * ts);
    if (fseeko(fp, (off_t)off, SEEK_SET) != 0 || fread(tmp.data(), ts, cnt, fp) != cnt) {
      fclose(fp);
      throw std::runtime_error(path + ": short read of '" + name + "'");
    }
    for (uint64_t e = 0; e < cnt; e++) dst[e] = (float)be_value(&tmp[e * ts], v.type);
  };
  if (!is_rec) {
    read_at(v.begin, n, out.data());
  } else {
    uint64_t recsize = 0, per = n / (f.numrecs ? f.numrecs : 1);
    int nrecvars = 0;
    for (size_t q = 0; q < f.vars.size(); q++) {
      const Var &w = f.vars[q];
      if (!w.dimids.empty() && f.dims[w.dimids[0]].len == 0) { recsize += w.vsize; nrecvars++; }
    }
    if (nrecvars == 1) recsize = per * ts;  // a single record variable is not padded
    for (uint64_t rec = 0; rec < f.numrecs; rec++) read_at(v.begin + rec * recsize, per, out.data() + rec * per);
  }
  fclose(fp);
  return out;
}

namespace {

std::vector<unsigned char> build_header(const File &f, const std::vector<uint64_t> &begins, uint32_t numrecs) {
  Writer w;
  w.b.insert(w.b.end(), {'C', 'D', 'F', (unsigned char)f.version});
  w.u32(numrecs);
  if (f.dims.empty()) { w.u32(0); w.u32(0); }
  else {
    w.u32(TAG_DIM);
    w.u32((uint32_t)f.dims.size());
    for (const Dim &d : f.dims) { w.name(d.name); w.u32((uint32_t)d.len); }
  }
  put_atts(w, f.gatts);
  if (f.vars.empty()) { w.u32(0); w.u32(0); }
  else {
    w.u32(TAG_VAR);
    w.u32((uint32_t)f.vars.size());
    for (size_t v = 0; v < f.vars.size(); v++) {
      const Var &var = f.vars[v];
      w.name(var.name);
      w.u32((uint32_t)var.dimids.size());
      for (int d : var.dimids) w.u32((uint32_t)d);
      put_atts(w, var.atts);
      w.u32((uint32_t)var.type);
      w.u32(var.vsize > 0xFFFFFFFCull ? 0xFFFFFFFFu : (uint32_t)var.vsize);
      if (f.version == 1) w.u32((uint32_t)begins[v]);
      else w.u64(begins[v]);
    }
  }
  return w.b;
}

// big-endian copy of n floats
void put_floats(std::vector<unsigned char> &tmp, const float *src, uint64_t n, uint64_t padded) {
  tmp.assign(padded, 0);
  for (uint64_t e = 0; e < n; e++) {
    uint32_t u;
    memcpy(&u, &src[e], 4);
    tmp[4 * e] = (unsigned char)(u >> 24);
    tmp[4 * e + 1] = (unsigned char)(u >> 16);
    tmp[4 * e + 2] = (unsigned char)(u >> 8);
    tmp[4 * e + 3] = (unsigned char)u;
  }
}

}  // namespace

void write(const std::string &path, File f, const std::vector<const float *> &data) {
  if (data.size() != f.vars.size()) throw std::runtime_error("netcdf write: one data array per variable");
  // sizes; all variables fixed-size float
  std::vector<uint64_t> nelem(f.vars.size());
  for (size_t v = 0; v < f.vars.size(); v++) {
    f.vars[v].type = FLOAT;
    uint64_t n = 1;
    for (int d : f.vars[v].dimids) {
      if (f.dims[d].len == 0) throw std::runtime_error("netcdf write: record variables go through RecordWriter");
      n *= f.dims[d].len;
    }
    nelem[v] = n;
    f.vars[v].vsize = pad4(n * 4);
  }
  std::vector<uint64_t> begins(f.vars.size(), 0);
  uint64_t off = build_header(f, begins, 0).size();
  for (size_t v = 0; v < f.vars.size(); v++) { begins[v] = off; off += f.vars[v].vsize; }
  if (f.version == 1 && off > 0x7FFFFFFFull) throw std::runtime_error("netcdf write: file too large for CDF-1");
  std::vector<unsigned char> h = build_header(f, begins, 0);
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) throw std::runtime_error("cannot create " + path);
  bool ok = fwrite(h.data(), 1, h.size(), fp) == h.size();
  std::vector<unsigned char> tmp;
  for (size_t v = 0; v < f.vars.size() && ok; v++) {
    put_floats(tmp, data[v], nelem[v], f.vars[v].vsize);
    ok = fwrite(tmp.data(), 1, tmp.size(), fp) == tmp.size();
  }
  if (fclose(fp) != 0 || !ok) throw std::runtime_error("netcdf write failed: " + path);
}

RecordWriter::RecordWriter(const std::string &path, File f) : path_(path) {
  nelem_.resize(f.vars.size());
  for (size_t v = 0; v < f.vars.size(); v++) {
    Var &var = f.vars[v];
    var.type = FLOAT;
    if (var.dimids.empty() || f.dims[var.dimids[0]].len != 0)
      throw std::runtime_error("netcdf record writer: every variable needs the record dimension first");
    uint64_t n = 1;
    for (size_t q = 1; q < var.dimids.size(); q++) n *= f.dims[var.dimids[q]].len;
    nelem_[v] = n;
    var.vsize = pad4(n * 4);  // per record
  }
  std::vector<uint64_t> begins(f.vars.size(), 0);
  uint64_t off = build_header(f, begins, 0).size();
  for (size_t v = 0; v < f.vars.size(); v++) { begins[v] = off; off += f.vars[v].vsize; }
  std::vector<unsigned char> h = build_header(f, begins, 0);
  fp_ = fopen(path.c_str(), "wb+");
  if (!fp_) throw std::runtime_error("cannot create " + path);
  if (fwrite(h.data(), 1, h.size(), fp_) != h.size()) throw std::runtime_error("netcdf write failed: " + path);
  fflush(fp_);
}

void RecordWriter::append(const std::vector<const float *> &data) {
  if (data.size() != nelem_.size()) throw std::runtime_error("netcdf append: one slab per variable");
  if (fseek(fp_, 0, SEEK_END) != 0) throw std::runtime_error("netcdf append failed: " + path_);
  std::vector<unsigned char> tmp;
  bool ok = true;
  for (size_t v = 0; v < nelem_.size() && ok; v++) {
    put_floats(tmp, data[v], nelem_[v], pad4(nelem_[v] * 4));
    ok = fwrite(tmp.data(), 1, tmp.size(), fp_) == tmp.size();
  }
  nrec_++;
  unsigned char q[4] = {(unsigned char)(nrec_ >> 24), (unsigned char)(nrec_ >> 16), (unsigned char)(nrec_ >> 8),
                        (unsigned char)nrec_};
  ok = ok && fseek(fp_, 4, SEEK_SET) == 0 && fwrite(q, 1, 4, fp_) == 4 && fflush(fp_) == 0;
  if (!ok) throw std::runtime_error("netcdf append failed: " + path_);
}

RecordWriter::~RecordWriter() {
  if (fp_) fclose(fp_);
}

}  // namespace nc
}  // namespace cgfd
