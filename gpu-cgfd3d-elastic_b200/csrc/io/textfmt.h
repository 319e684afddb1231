// textfmt.h -- the reference's text inputs (.src source file, station list) and the SAC
// seismogram output, for the drop-in CLI.
#pragma once

#include <string>
#include <vector>

#include "cgfd_b200.h"

namespace cgfd {
namespace fmt {

// Parsed .src file (src_t.cu:205-611); desc() points into the owned arrays.
struct SourceFile {
  std::string evtnm;
  cgfd_source_desc d{};
  std::vector<float> loc, t_start, coefs, cmp, cmp_values;
  std::vector<int> wavelet;
  const cgfd_source_desc &desc();
};
SourceFile read_source_file(const std::string &path);

// Parsed station list (io_funcs.cu:52-80).
struct StationFile {
  std::vector<std::string> names;
  std::vector<int> flag_coord, flag_depth;
  std::vector<float> loc;
  cgfd_station_desc d{};
  const cgfd_station_desc &desc();
};
StationFile read_station_file(const std::string &path);

// Layer model file of any elastic media type (read_interface_file,
// src/media/media_read_file.cpp:22-700; lines starting with '#' and empty lines skipped, then
// whitespace-separated tokens): the media type name (elastic_isotropic, elastic_vti_prem,
// elastic_vti_thomsen, elastic_vti_cij, elastic_tti_thomsen, elastic_tti_bond,
// elastic_aniso_cij), number of interfaces, "NX NY MINX MINY DX DY", then per interface and
// mesh point the elevation and value / gradient / power of every parameter of the type.
// media() (every type) and desc() (elastic_isotropic) point into the arrays.
struct LayerFile {
  int type = 0;  // CGFD_LAYER_*
  int ni = 0, nx = 0, ny = 0, npar = 0;
  float x0 = 0, y0 = 0, dx = 0, dy = 0;
  std::vector<float> elevation;  // [ni][ny][nx]
  std::vector<float> param;      // [npar][3][ni][ny][nx]
  cgfd_layer_model d{};
  cgfd_layer_media m{};
  const cgfd_layer_model &desc();
  const cgfd_layer_media &media();
};
LayerFile read_layer_file(const std::string &path);

// Grid media file (read_grid_file, media_read_file.cpp:670-1266) of the elastic types: the type
// name, the number of layers, the surfaces of each layer, "NX NY MINX MINY DX DY", then per
// surface and mesh point (x fastest) the elevation and the type's parameters; a layer's last
// surface must lie on the next layer's first (checkGridData, :1242-1266).
struct GridFile {
  int type = 0, npar = 0;  // CGFD_LAYER_*
  std::vector<int> ngz;
  int ni = 0, nx = 0, ny = 0;
  float x0 = 0, y0 = 0, dx = 0, dy = 0;
  std::vector<float> elevation;  // [ni][ny][nx]
  std::vector<float> param;      // [npar][ni][ny][nx]
  cgfd_grid_media d{};
  const cgfd_grid_media &desc();
};
GridFile read_grid_file(const std::string &path);

// One-component SAC file with the header fields the reference sets (sacLib.cu:8-100):
// delta, b = 0, e = delta*(npts-1), npts, nvhdr = 6, iftype = ITIME, leven = 1, station
// and event positions; every other field "undefined" (-12345).
void write_sac(const std::string &path, const float *data, int npts, float delta, float stla, float stlo,
               float stel, float stdp, float evla = 0.f, float evlo = 0.f, float evel = 0.f, float evdp = 0.f);

}  // namespace fmt
}  // namespace cgfd
