// textfmt.cpp -- .src / station-list readers and SAC writer.
#include "textfmt.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace cgfd {
namespace fmt {

namespace {

// next line that is not empty and does not start with '#' (io_funcs.cu:2130-2154)
struct Lines {
  std::ifstream f;
  std::string path;
  explicit Lines(const std::string &p) : f(p), path(p) {
    if (!f) throw std::runtime_error("cannot open " + p);
  }
  std::string next() {
    std::string ln;
    while (std::getline(f, ln)) {
      if (!ln.empty() && ln.back() == '\r') ln.pop_back();
      if (ln.empty() || ln[0] == '#') continue;
      return ln;
    }
    throw std::runtime_error(path + ": unexpected end of file");
  }
};

std::vector<float> numbers(const std::string &ln, size_t max_n) {
  std::istringstream ss(ln);
  std::vector<float> v;
  float x;
  while (v.size() < max_n && ss >> x) v.push_back(x);
  return v;
}

int wavelet_id(const std::string &name) {
  if (name == "ricker") return CGFD_WAVELET_RICKER;
  if (name == "gaussian") return CGFD_WAVELET_GAUSSIAN;
  if (name == "ricker_deriv") return CGFD_WAVELET_RICKER_DERIV;
  if (name == "gaussian_deriv") return CGFD_WAVELET_GAUSSIAN_DERIV;
  if (name == "klauder") return CGFD_WAVELET_KLAUDER;
  throw std::runtime_error("wavelet '" + name + "' is not implemented");
}

}  // namespace

const cgfd_source_desc &SourceFile::desc() {
  d.loc = loc.data();
  d.t_start = t_start.data();
  d.wavelet = wavelet.empty() ? nullptr : wavelet.data();
  d.wavelet_coefs = coefs.empty() ? nullptr : coefs.data();
  d.cmp = cmp.empty() ? nullptr : cmp.data();
  d.cmp_values = cmp_values.empty() ? nullptr : cmp_values.data();
  return d;
}

SourceFile read_source_file(const std::string &path) {
  Lines in(path);
  SourceFile s;
  s.evtnm = in.next();
  int n = (int)numbers(in.next(), 1).at(0);
  if (n <= 0) throw std::runtime_error(path + ": number of sources must be > 0");
  std::vector<float> w = numbers(in.next(), 3);
  s.d.num = n;
  s.d.stf_given = (int)w.at(0);
  if (s.d.stf_given == 0) s.d.stf_length = w.at(1);
  else if (s.d.stf_given == 1) { s.d.stf_dt = w.at(1); s.d.stf_nt = (int)w.at(2); }
  else throw std::runtime_error(path + ": stf_given must be 0 or 1");
  w = numbers(in.next(), 2);
  s.d.cmp_type = (int)w.at(0);
  s.d.mechanism_type = (int)w.at(1);
  w = numbers(in.next(), 2);
  s.d.loc_coord_type = (int)w.at(0);
  s.d.loc_3dim = (int)w.at(1);
  s.loc.resize(3 * n);
  for (int i = 0; i < n; i++) {
    w = numbers(in.next(), 3);
    for (int a = 0; a < 3; a++) s.loc[3 * i + a] = w.at(a);
  }
  s.t_start.resize(n);
  int c0 = s.d.cmp_type == 2 ? 3 : 0;
  int nc = s.d.cmp_type == 1 ? 3 : (s.d.cmp_type == 2 ? 6 : 9);
  // values missing on a line keep what the previous source left (sscanf into persistent
  // variables, src_t.cu:491-507)
  float prev[9] = {0}, prevc[10] = {0};
  if (s.d.stf_given == 0) {
    s.wavelet.resize(n);
    s.coefs.assign(10 * n, 0.f);
    s.cmp.assign(9 * n, 0.f);
    for (int i = 0; i < n; i++) {
      std::istringstream ss(in.next());
      std::string name;
      ss >> s.t_start[i] >> name;
      s.wavelet[i] = wavelet_id(name);
      float x;
      for (int c = 0; c < 10 && ss >> x; c++) prevc[c] = x;
      memcpy(&s.coefs[10 * i], prevc, sizeof(prevc));
      w = numbers(in.next(), nc);
      for (size_t c = 0; c < w.size(); c++) prev[c0 + c] = w[c];
      memcpy(&s.cmp[9 * i], prev, sizeof(prev));
    }
  } else {
    s.cmp_values.assign((size_t)n * s.d.stf_nt * 9, 0.f);
    for (int i = 0; i < n; i++) {
      s.t_start[i] = numbers(in.next(), 1).at(0);
      for (int t = 0; t < s.d.stf_nt; t++) {
        w = numbers(in.next(), nc);
        for (size_t c = 0; c < w.size(); c++) s.cmp_values[((size_t)i * s.d.stf_nt + t) * 9 + c0 + c] = w[c];
      }
    }
  }
  s.desc();
  return s;
}

const cgfd_station_desc &StationFile::desc() {
  d.num = (int)names.size();
  d.flag_coord = flag_coord.data();
  d.flag_depth = flag_depth.data();
  d.loc = loc.data();
  return d;
}

StationFile read_station_file(const std::string &path) {
  Lines in(path);
  StationFile s;
  int n = (int)numbers(in.next(), 1).at(0);
  for (int i = 0; i < n; i++) {
    std::istringstream ss(in.next());
    std::string name;
    int fc = 0, fd = 0;
    float x = 0, y = 0, z = 0;
    if (!(ss >> name >> fc >> fd >> x >> y >> z)) throw std::runtime_error(path + ": malformed station line");
    s.names.push_back(name);
    s.flag_coord.push_back(fc);
    s.flag_depth.push_back(fd);
    s.loc.insert(s.loc.end(), {x, y, z});
  }
  s.desc();
  return s;
}

LayerFile read_layer_file(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::stringstream body;
  std::string ln;
  while (std::getline(in, ln)) {
    if (ln.empty() || ln[0] == '#' || ln[0] == '\r') continue;
    body << ln << "\n";
  }
  LayerFile L;
  std::string type;
  if (!(body >> type)) throw std::runtime_error(path + ": no media type");
  static const struct { const char *name; int type, npar; } kTypes[] = {
      {"acoustic_isotropic", CGFD_LAYER_ACOUSTIC_ISO, 2},
      {"elastic_isotropic", CGFD_LAYER_ELASTIC_ISO, 3},  {"elastic_vti_prem", CGFD_LAYER_VTI_PREM, 6},
      {"elastic_vti_thomsen", CGFD_LAYER_VTI_THOMSEN, 6}, {"elastic_vti_cij", CGFD_LAYER_VTI_CIJ, 6},
      {"elastic_tti_thomsen", CGFD_LAYER_TTI_THOMSEN, 8}, {"elastic_tti_bond", CGFD_LAYER_TTI_BOND, 8},
      {"elastic_aniso_cij", CGFD_LAYER_ANISO_CIJ, 22}};
  for (const auto &t : kTypes)
    if (type == t.name) { L.type = t.type; L.npar = t.npar; }
  if (!L.type)
    throw std::runtime_error(path + ": media type '" + type + "' is not on this path (acoustic and elastic types)");
  if (!(body >> L.ni) || L.ni < 1) throw std::runtime_error(path + ": number of interfaces missing or < 1");
  if (!(body >> L.nx >> L.ny >> L.x0 >> L.y0 >> L.dx >> L.dy) || L.nx < 2 || L.ny < 2)
    throw std::runtime_error(path + ": interface mesh line must be NX NY MINX MINY DX DY with NX, NY >= 2");
  const size_t n = (size_t)L.ni * L.nx * L.ny;
  L.elevation.resize(n);
  L.param.resize((size_t)L.npar * 3 * n);
  for (size_t p = 0; p < n; p++) {
    if (!(body >> L.elevation[p])) throw std::runtime_error(path + ": insufficient data");
    for (int q = 0; q < 3 * L.npar; q++)
      if (!(body >> L.param[(size_t)q * n + p])) throw std::runtime_error(path + ": insufficient data");
  }
  return L;
}

GridFile read_grid_file(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  GridFile G;
  std::string type;
  if (!(in >> type)) throw std::runtime_error(path + ": no media type");
  static const struct { const char *name; int type, npar; } kTypes[] = {
      {"elastic_isotropic", CGFD_LAYER_ELASTIC_ISO, 3},     {"elastic_vti_prem", CGFD_LAYER_VTI_PREM, 6},
      {"elastic_vti_thomsen", CGFD_LAYER_VTI_THOMSEN, 6}, {"elastic_vti_cij", CGFD_LAYER_VTI_CIJ, 6},
      {"elastic_tti_thomsen", CGFD_LAYER_TTI_THOMSEN, 8}, {"elastic_aniso_cij", CGFD_LAYER_ANISO_CIJ, 22}};
  for (const auto &t : kTypes)
    if (type == t.name) { G.type = t.type; G.npar = t.npar; }
  if (!G.type) throw std::runtime_error(path + ": grid media of type '" + type + "' are not on this path");
  int nl = 0;
  if (!(in >> nl) || nl < 1) throw std::runtime_error(path + ": number of layers missing or < 1");
  for (int l = 0; l < nl; l++) {
    int ng = 0;
    if (!(in >> ng) || ng < 1) throw std::runtime_error(path + ": surfaces of a layer missing or < 1");
    G.ngz.push_back(ng);
    G.ni += ng;
  }
  if (!(in >> G.nx >> G.ny >> G.x0 >> G.y0 >> G.dx >> G.dy) || G.nx < 2 || G.ny < 2)
    throw std::runtime_error(path + ": mesh line must be NX NY MINX MINY DX DY with NX, NY >= 2");
  const size_t sl = (size_t)G.nx * G.ny, n = (size_t)G.ni * sl;
  G.elevation.resize(n);
  G.param.resize((size_t)G.npar * n);
  for (size_t p = 0; p < n; p++) {
    if (!(in >> G.elevation[p])) throw std::runtime_error(path + ": insufficient data");
    for (int q = 0; q < G.npar; q++)
      if (!(in >> G.param[(size_t)q * n + p])) throw std::runtime_error(path + ": insufficient data");
  }
  int s = 0;
  for (int l = 0; l + 1 < nl; l++) {
    s += G.ngz[l];
    for (size_t p = 0; p < sl; p++)
      if (G.elevation[(size_t)(s - 1) * sl + p] != G.elevation[(size_t)s * sl + p])
        throw std::runtime_error(path + ": the last elevations of layer " + std::to_string(l) +
                                 " must equal the first elevations of layer " + std::to_string(l + 1));
  }
  return G;
}

const cgfd_grid_media &GridFile::desc() {
  d.type = type;
  d.num_layers = (int)ngz.size();
  d.ngz = ngz.data();
  d.nx = nx; d.ny = ny;
  d.x0 = x0; d.y0 = y0; d.dx = dx; d.dy = dy;
  d.elevation = elevation.data();
  d.param = param.data();
  return d;
}

const cgfd_layer_model &LayerFile::desc() {
  const size_t n = (size_t)ni * nx * ny;
  d.num_interfaces = ni; d.nx = nx; d.ny = ny;
  d.x0 = x0; d.y0 = y0; d.dx = dx; d.dy = dy;
  d.elevation = elevation.data();
  const float **dst[9] = {&d.rho, &d.rho_grad, &d.rho_pow, &d.vp, &d.vp_grad, &d.vp_pow, &d.vs, &d.vs_grad, &d.vs_pow};
  for (int q = 0; q < 9 && q < 3 * npar; q++) *dst[q] = param.data() + (size_t)q * n;
  return d;
}

const cgfd_layer_media &LayerFile::media() {
  m.type = type;
  m.num_interfaces = ni; m.nx = nx; m.ny = ny;
  m.x0 = x0; m.y0 = y0; m.dx = dx; m.dy = dy;
  m.elevation = elevation.data();
  m.param = param.data();
  return m;
}

void write_sac(const std::string &path, const float *data, int npts, float delta, float stla, float stlo, float stel,
               float stdp, float evla, float evlo, float evel, float evdp) {
  // SAC binary header: 70 floats, 40 ints (incl. 5 logicals), 192 bytes of text (632 bytes)
  float fh[70];
  int ih[40];
  char ch[192];
  for (float &x : fh) x = -12345.0f;
  for (int &x : ih) x = -12345;
  // 23 text fields: kstnm(8) kevnm(16) and 21 more of 8 bytes
  for (int q = 0; q < 23; q++) {
    int len = q == 1 ? 16 : 8;
    int off = q == 0 ? 0 : (q == 1 ? 8 : 24 + (q - 2) * 8);
    memset(ch + off, 0, len);
    memcpy(ch + off, "-12345  ", 8);
  }
  // kstnm and kcmpnm are "-12345" (sacLib.cu:55-56)
  memset(ch + 0, 0, 8);
  memcpy(ch + 0, "-12345", 6);
  memset(ch + 160, 0, 8);
  memcpy(ch + 160, "-12345", 6);
  fh[0] = delta;                 // delta
  fh[5] = 0.0f;                  // b
  fh[6] = delta * (npts - 1);    // e
  fh[31] = stla; fh[32] = stlo; fh[33] = stel; fh[34] = stdp;
  fh[35] = evla; fh[36] = evlo; fh[37] = evel; fh[38] = evdp;
  fh[57] = 0.0f; fh[58] = 0.0f;  // cmpaz, cmpinc
  ih[6] = 6;                     // nvhdr
  ih[9] = npts;                  // npts
  ih[15] = 1;                    // iftype = ITIME
  ih[35] = 1;                    // leven
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) throw std::runtime_error("cannot create " + path);
  bool ok = fwrite(fh, 4, 70, fp) == 70 && fwrite(ih, 4, 40, fp) == 40 && fwrite(ch, 1, 192, fp) == 192 &&
            fwrite(data, 4, npts, fp) == (size_t)npts;
  if (fclose(fp) != 0 || !ok) throw std::runtime_error("write failed: " + path);
}

}  // namespace fmt
}  // namespace cgfd
