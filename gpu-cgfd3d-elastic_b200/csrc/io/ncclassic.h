// ncclassic.h -- NetCDF classic format (CDF-1, and CDF-2 "64-bit offset") reader and writer,
// written from the public file-format specification. Enough for the grid, metric, medium and
// snapshot files of the reference (fixed-size float variables with int/float attributes;
// the reader also handles record variables).
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace cgfd {
namespace nc {

enum Type { BYTE = 1, CHAR = 2, SHORT = 3, INT = 4, FLOAT = 5, DOUBLE = 6 };

struct Dim {
  std::string name;
  uint64_t len;  // 0 = record (unlimited) dimension
};

struct Att {
  std::string name;
  int type;
  std::vector<double> num;  // numeric values
  std::string text;         // CHAR attributes
};

struct Var {
  std::string name;
  std::vector<int> dimids;
  std::vector<Att> atts;
  int type = FLOAT;
  uint64_t vsize = 0, begin = 0;
};

struct File {
  int version = 2;  // 1 = CDF-1, 2 = CDF-2
  uint64_t numrecs = 0;
  std::vector<Dim> dims;
  std::vector<Att> gatts;
  std::vector<Var> vars;

  int find_var(const std::string &name) const;
  const Att *find_gatt(const std::string &name) const;
  // shape of a variable (record dimension -> numrecs)
  std::vector<uint64_t> shape(int varid) const;
};

// Reads the header of `path`.
File read_header(const std::string &path);

// Reads a whole variable, converted to float (FLOAT/DOUBLE/INT/SHORT/BYTE supported).
std::vector<float> read_var(const std::string &path, const File &f, const std::string &name);

// Writes `f` (dims, global atts, fixed-size float variables) with the given data arrays,
// one per variable in f.vars order. Throws on I/O errors.
void write(const std::string &path, File f, const std::vector<const float *> &data);

// A file of float record variables (every variable's first dimension is the record
// dimension, length 0 in f.dims): the header goes out at construction, append() adds one
// record (one slab per variable, f.vars order) and rewrites numrecs, so the file is valid
// after every record (like nc_put_vara on an NC_UNLIMITED dimension).
class RecordWriter {
 public:
  RecordWriter(const std::string &path, File f);
  ~RecordWriter();
  RecordWriter(const RecordWriter &) = delete;
  RecordWriter &operator=(const RecordWriter &) = delete;
  void append(const std::vector<const float *> &data);
  uint64_t records() const { return nrec_; }

 private:
  FILE *fp_ = nullptr;
  std::string path_;
  std::vector<uint64_t> nelem_;
  uint64_t nrec_ = 0;
};

}  // namespace nc
}  // namespace cgfd
