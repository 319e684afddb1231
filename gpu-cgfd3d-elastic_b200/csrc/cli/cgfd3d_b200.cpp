// cgfd3d_b200.cpp -- drop-in command line driver: `cgfd3d_b200 <par.json> <gpu_id>`.
//
// Reproduces the observable behaviour of the reference's main (main_curv_col_el_3d.cu:22-853)
// for the elastic time-loop path on one GPU: reads the same parameter file keys, grid /
// metric / medium NetCDF files, .src source file and station list, checks the time step
// (FP64), runs the B200 time loop through the C ABI and writes the same SAC files
// (<output_dir>/<station>.<Vx..Txy>.sac, plus <station>.E**.sac strain for isotropic media;
// <station>.<Vx Vy Vz P>.sac for acoustic media), line receivers, slices and snapshots, and
// with a free surface the peak ground motion file PG_V_A_D_px0_py0_pz0.nc. Media come from
// media_*.nc files, or from layer files, grid files or binary models discretised on the GPU. Options outside this path (MPI
// decomposition, ablexp, visco-elastic Q volumes from one-component media files) are rejected
// with a message; visco-elastic media (visco_type gmb) are read through the media import.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <memory>
#include <string>
#include <vector>

#include "cgfd_b200.h"
#include "io/json.h"
#include "io/ncclassic.h"
#include "io/textfmt.h"

using cgfd::json::Value;

namespace {

const char *kFnamePart = "px0_py0_pz0";  // blk_set_output (blk_t.cu:54) for one rank
const char *kCmpNames[9] = {"Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Tyz", "Txz", "Txy"};
// Output components of the medium (wav_init / wav_ac_init, wav_t.cu:14-250): the 9 elastic
// ones, or Vx Vy Vz P for acoustic media (P in the device's Txx slot).
const char *kAcNames[4] = {"Vx", "Vy", "Vz", "P"};
int g_ncmp = 9;
const char *const *g_names = kCmpNames;

[[noreturn]] void fail(const std::string &m) { throw std::runtime_error(m); }

const Value &need(const Value &o, const char *key) {
  const Value *v = o.get(key);
  if (!v) fail(std::string("missing key '") + key + "'");
  return *v;
}

struct Grid {
  int ni, nj, nk;
  size_t nx, ny, nz, siz;
  size_t at(int i, int j, int k) const { return (size_t)(i + 3) + (size_t)(j + 3) * nx + (size_t)(k + 3) * nx * ny; }
};

// physical-point float variable [nk][nj][ni] -> reference layout field (ghosts untouched)
void put_physical(const Grid &g, const std::vector<float> &v, float *field) {
  if (v.size() != (size_t)g.ni * g.nj * g.nk) fail("variable size does not match the grid");
  size_t n = 0;
  for (int k = 0; k < g.nk; k++)
    for (int j = 0; j < g.nj; j++)
      for (int i = 0; i < g.ni; i++) field[g.at(i, j, k)] = v[n++];
}

void import_vars(const std::string &path, const Grid &g, const std::vector<std::string> &names, float *dst) {
  cgfd::nc::File f = cgfd::nc::read_header(path);
  for (size_t c = 0; c < names.size(); c++) {
    std::vector<float> v = cgfd::nc::read_var(path, f, names[c]);
    put_physical(g, v, dst + c * g.siz);
  }
}

// One "snapshot" entry of the par file, located in the grid like io_snapshot_locate
// (io_funcs.cu:790-929): 1-based start in the file, indices outside the physical grid dropped.
struct Snap {
  std::string name;
  int start[3], count[3], incre[3];   // 0-based first inner index, inner count, stride
  int first_in_nc[3];                 // position of `start` in the requested index list
  int it1, dit, vel, stress, strain;
  std::unique_ptr<cgfd::nc::RecordWriter> w;
};

Snap parse_snapshot(const Value &e, const Grid &g) {
  Snap s;
  s.name = need(e, "name").as_str();
  const Value &st = need(e, "grid_index_start"), &ct = need(e, "grid_index_count"), &ic = need(e, "grid_index_incre");
  if (st.arr.size() != 3 || ct.arr.size() != 3 || ic.arr.size() != 3) fail("snapshot index arrays need 3 entries");
  const int n[3] = {g.ni, g.nj, g.nk};
  for (int a = 0; a < 3; a++) {
    const int g1 = st.arr[a].as_int() - 1, cnt = ct.arr[a].as_int(), inc = ic.arr[a].as_int();
    if (inc < 1) fail("snapshot " + s.name + ": grid_index_incre must be >= 1");
    int first = -1, num = 0, pos = 0;
    for (int q = 0; q < cnt; q++) {
      const int gi = g1 + q * inc;
      if (gi >= 0 && gi < n[a]) {
        if (first < 0) { first = gi; pos = q; }
        num++;
      }
      if (gi > n[a] - 1) break;
    }
    if (num == 0) fail("snapshot " + s.name + " lies outside the grid");
    s.start[a] = first;
    s.count[a] = num;
    s.incre[a] = inc;
    s.first_in_nc[a] = pos;
  }
  s.it1 = need(e, "time_index_start").as_int();
  s.dit = need(e, "time_index_incre").as_int();
  if (s.dit < 1) fail("snapshot " + s.name + ": time_index_incre must be >= 1");
  s.vel = e.get("save_velocity") ? e.get("save_velocity")->as_int() : 0;
  s.stress = e.get("save_stress") ? e.get("save_stress")->as_int() : 0;
  s.strain = e.get("save_strain") ? e.get("save_strain")->as_int() : 0;
  return s;
}

// io_snap_nc_create (io_funcs.cu:931-1047): time (unlimited), k, j, i; time, then the
// requested groups Vx Vy Vz / Txx Tyy Tzz Txz Tyz Txy / Exx Eyy Ezz Exz Eyz Exy.
void open_snapshot(Snap &s, const std::string &out) {
  cgfd::nc::File f;
  f.version = 1;
  f.dims = {{"time", 0}, {"k", (uint64_t)s.count[2]}, {"j", (uint64_t)s.count[1]}, {"i", (uint64_t)s.count[0]}};
  auto var = [&](const char *name, bool scalar) {
    cgfd::nc::Var v;
    v.name = name;
    v.dimids = scalar ? std::vector<int>{0} : std::vector<int>{0, 1, 2, 3};
    f.vars.push_back(v);
  };
  var("time", true);
  if (s.vel == 1) for (const char *n : {"Vx", "Vy", "Vz"}) var(n, false);
  if (g_ncmp == 4) {  // acoustic (io_snap_nc_create_ac, io_funcs.cu:1258-1350): the pressure as "Tii"
    if (s.strain == 1) fail("snapshot strain of acoustic media is not computed (io_snap_nc_put_ac leaves it unwritten)");
    if (s.stress == 1) var("Tii", false);
  } else {
    if (s.stress == 1) for (const char *n : {"Txx", "Tyy", "Tzz", "Txz", "Tyz", "Txy"}) var(n, false);
    if (s.strain == 1) for (const char *n : {"Exx", "Eyy", "Ezz", "Exz", "Eyz", "Exy"}) var(n, false);
  }
  f.gatts.push_back({"first_index_to_snapshot_output", cgfd::nc::INT,
                     {(double)s.first_in_nc[0], (double)s.first_in_nc[1], (double)s.first_in_nc[2]}, ""});
  f.gatts.push_back({"first_index_in_this_thread_with_ghosts", cgfd::nc::INT,
                     {(double)s.start[0] + 3, (double)s.start[1] + 3, (double)s.start[2] + 3}, ""});
  f.gatts.push_back({"index_stride_in_this_thread", cgfd::nc::INT,
                     {(double)s.incre[0], (double)s.incre[1], (double)s.incre[2]}, ""});
  f.gatts.push_back({"coords_of_mpi_topo", cgfd::nc::INT, {0.0, 0.0, 0.0}, ""});
  s.w.reset(new cgfd::nc::RecordWriter(out + "/" + s.name + "_" + kFnamePart + ".nc", f));
}

// io_snap_nc_put (io_funcs.cu:1049-1256): at step it (state at the start of the step)
bool snapshot_due(const Snap &s, int it, int nt_total) {
  return it >= s.it1 && (it - s.it1) % s.dit == 0 && (it - s.it1) / s.dit <= (nt_total - s.it1) / s.dit;
}

void put_snapshot(Snap &s, cgfd_problem *p, const Grid &g, const std::vector<float> &medium, int iso, float time) {
  const size_t n = (size_t)s.count[0] * s.count[1] * s.count[2];
  std::vector<float> box(9 * n);
  if (cgfd_get_wavefield_box(p, 0, s.start, s.count, s.incre, box.data()))
    fail(std::string("snapshot: ") + cgfd_last_error());
  // device component order Vx Vy Vz Txx Tyy Tzz Tyz Txz Txy; the file's stress order puts Txz
  // before Tyz
  const float *c[9];
  for (int q = 0; q < 9; q++) c[q] = box.data() + q * n;
  std::vector<const float *> data = {&time};
  if (s.vel == 1) data.insert(data.end(), {c[0], c[1], c[2]});
  if (s.stress == 1 && g_ncmp == 4) data.push_back(c[3]);  // acoustic: P (io_snap_nc_put_ac)
  else if (s.stress == 1) data.insert(data.end(), {c[3], c[4], c[5], c[7], c[6], c[8]});
  std::vector<float> E;
  if (s.strain == 1) {
    if (!iso) fail("snapshot strain is computed for elastic_iso media only (io_snap_stress_to_strain_eliso)");
    // io_snap_stress_to_strain_eliso (io_funcs.cu:1462-1567)
    E.resize(6 * n);
    size_t m = 0;
    for (int kk = 0; kk < s.count[2]; kk++)
      for (int jj = 0; jj < s.count[1]; jj++)
        for (int ii = 0; ii < s.count[0]; ii++, m++) {
          const size_t at = g.at(s.start[0] + ii * s.incre[0], s.start[1] + jj * s.incre[1], s.start[2] + kk * s.incre[2]);
          const float lam = medium[g.siz + at], mu = medium[2 * g.siz + at];
          const float E1 = (float)((lam + mu) / (mu * (3.0 * lam + 2.0 * mu)));
          const float E2 = (float)(-lam / (2.0 * mu * (3.0 * lam + 2.0 * mu)));
          const float E3 = (float)(1.0 / mu);
          const float E0 = E2 * (c[3][m] + c[4][m] + c[5][m]);
          E[0 * n + m] = E0 - (E2 - E1) * c[3][m];
          E[1 * n + m] = E0 - (E2 - E1) * c[4][m];
          E[2 * n + m] = E0 - (E2 - E1) * c[5][m];
          E[3 * n + m] = 0.5f * E3 * c[7][m];  // Exz
          E[4 * n + m] = 0.5f * E3 * c[6][m];  // Eyz
          E[5 * n + m] = 0.5f * E3 * c[8][m];  // Exy
        }
    for (int q = 0; q < 6; q++) data.push_back(E.data() + q * n);
  }
  s.w->append(data);
}

// One receiver of a "receiver_line" entry inside the grid (io_line_locate, io_funcs.cu:300-414):
// point `seq` of the line at physical index start + seq * incre.
struct LinePoint {
  std::string line;
  int seq, i, j, k;
};

std::vector<LinePoint> parse_lines(const Value *lv, const Grid &g) {
  std::vector<LinePoint> pts;
  if (!lv) return pts;
  for (const Value &e : lv->arr) {
    const std::string name = need(e, "name").as_str();
    const Value &st = need(e, "grid_index_start"), &ic = need(e, "grid_index_incre");
    if (st.arr.size() != 3 || ic.arr.size() != 3) fail("receiver_line " + name + ": index arrays need 3 entries");
    const int cnt = need(e, "grid_index_count").as_int();
    for (int n = 0; n < cnt; n++) {
      int q[3];
      for (int a = 0; a < 3; a++) q[a] = st.arr[a].as_int() - 1 + n * ic.arr[a].as_int();  // 1-based in the file
      if (q[0] >= 0 && q[0] < g.ni && q[1] >= 0 && q[1] < g.nj && q[2] >= 0 && q[2] < g.nk)
        pts.push_back({name, n, q[0], q[1], q[2]});
    }
  }
  return pts;
}

// The x / y / z slices of the "slice" entry inside the grid (io_slice_locate,
// io_funcs.cu:418-528), each a NetCDF file of record variables on an unlimited time dimension
// (io_slice_nc_create, io_funcs.cu:531-664): slicex_i<gi+1>_<part>.nc with dims (time, k, j),
// slicey_j<gj+1> (time, k, i), slicez_k<gk+1> (time, j, i); variable "time" and the medium's
// components (9 elastic, 4 acoustic).
struct Slices {
  std::vector<int> idx[3];
  std::vector<std::unique_ptr<cgfd::nc::RecordWriter>> files[3];
};

Slices open_slices(const Value *sv, const Grid &g, const std::string &out) {
  Slices S;
  if (!sv) return S;
  const char *keys[3] = {"x_index", "y_index", "z_index"};
  const int n[3] = {g.ni, g.nj, g.nk};
  const char *tag[3] = {"slicex_i", "slicey_j", "slicez_k"};
  const char *att[3] = {"i_index_with_ghosts_in_this_thread", "j_index_with_ghosts_in_this_thread",
                        "k_index_with_ghosts_in_this_thread"};
  for (int a = 0; a < 3; a++) {
    const Value *v = sv->get(keys[a]);
    if (!v) continue;
    for (const Value &e : v->arr) {
      const int gi = e.as_int() - 1;
      if (gi < 0 || gi >= n[a]) continue;
      S.idx[a].push_back(gi);
      cgfd::nc::File f;
      f.version = 1;  // NC_CLOBBER: classic format
      const std::string d1 = a == 2 ? "j" : "k", d2 = a == 0 ? "j" : "i";
      f.dims = {{"time", 0}, {d1, (uint64_t)(a == 2 ? g.nj : g.nk)}, {d2, (uint64_t)(a == 0 ? g.nj : g.ni)}};
      cgfd::nc::Var tv;
      tv.name = "time";
      tv.dimids = {0};
      f.vars.push_back(tv);
      for (int c = 0; c < g_ncmp; c++) {
        cgfd::nc::Var v3;
        v3.name = g_names[c];
        v3.dimids = {0, 1, 2};
        f.vars.push_back(v3);
      }
      f.gatts.push_back({att[a], cgfd::nc::INT, {(double)(gi + 3)}, ""});
      f.gatts.push_back({"coords_of_mpi_topo", cgfd::nc::INT, {0.0, 0.0, 0.0}, ""});
      S.files[a].emplace_back(new cgfd::nc::RecordWriter(
          out + "/" + tag[a] + std::to_string(gi + 1) + "_" + kFnamePart + ".nc", f));
    }
  }
  return S;
}

// Appends the slices of step `it` (io_slice_nc_put: time = it * dt + t0, then each component).
void put_slices(Slices &S, cgfd_problem *p, const Grid &g, int it, float time, std::vector<float> &buf) {
  const size_t plane[3] = {(size_t)g.nk * g.nj, (size_t)g.nk * g.ni, (size_t)g.nj * g.ni};
  size_t total = 0;
  for (int a = 0; a < 3; a++) total += S.idx[a].size() * 9 * plane[a];
  buf.resize(total);
  if (cgfd_get_slices(p, 0, it, buf.data())) fail(std::string("slices: ") + cgfd_last_error());
  size_t off = 0;
  for (int a = 0; a < 3; a++)
    for (size_t s = 0; s < S.idx[a].size(); s++) {
      std::vector<const float *> data = {&time};
      for (int c = 0; c < g_ncmp; c++) data.push_back(buf.data() + off + c * plane[a]);
      S.files[a][s]->append(data);
      off += 9 * plane[a];
    }
}

void mkdirs(const std::string &d) {
  std::string cur;
  for (size_t p = 0; p <= d.size(); p++) {
    if (p == d.size() || d[p] == '/') {
      if (!cur.empty()) mkdir(cur.c_str(), 0755);
    }
    if (p < d.size()) cur += d[p];
  }
}

int run(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: cgfd3d_b200 <par_file> <gpu_id>\n");
    return 1;
  }
  Value par = cgfd::json::parse_file(argv[1]);
  int gpu = atoi(argv[2]);

  Grid g;
  g.ni = need(par, "number_of_total_grid_points_x").as_int();
  g.nj = need(par, "number_of_total_grid_points_y").as_int();
  g.nk = need(par, "number_of_total_grid_points_z").as_int();
  g.nx = g.ni + 6; g.ny = g.nj + 6; g.nz = g.nk + 6;
  g.siz = g.nx * g.ny * g.nz;
  if (const Value *v = par.get("number_of_mpiprocs_x"))
    if (v->as_int() != 1) fprintf(stderr, "note: number_of_mpiprocs_x ignored (one GPU, one block)\n");

  // ---- time (par_t.cu:150-200)
  double dt = -1.0, twin = -1.0, t0 = 0.0;
  int nsteps = -1, check = 1;
  if (const Value *v = par.get("size_of_time_step")) dt = v->as_num();
  if (const Value *v = par.get("number_of_time_steps")) nsteps = v->as_int();
  if (const Value *v = par.get("time_window_length")) twin = v->as_num();
  if (const Value *v = par.get("time_start")) t0 = v->as_num();
  if (const Value *v = par.get("check_stability")) check = v->as_int();
  if (dt < 0.0 && twin < 0.0) fail("at least one of size_of_time_step / time_window_length must be > 0");
  if (dt > 0.0) {
    if (nsteps < 0 && twin < 0.0) fail("both number_of_time_steps and time_window_length are missing");
    if (nsteps < 0) nsteps = (int)(twin / dt + 0.5);
    twin = dt * nsteps;
  }
  int nt_total = nsteps + 1;

  // ---- boundaries (par_t.cu:218-371)
  cgfd_problem_desc d;
  memset(&d, 0, sizeof(d));
  const char *bnames[3][2] = {{"boundary_x_left", "boundary_x_right"},
                              {"boundary_y_front", "boundary_y_back"},
                              {"boundary_z_bottom", "boundary_z_top"}};
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) {
      const Value *b = par.get(bnames[a][s]);
      if (!b) continue;
      if (const Value *c = b->get("cfspml")) {
        d.pml[a][s].enable = 1;
        d.pml[a][s].num_layers = need(*c, "number_of_layers").as_int();
        d.pml[a][s].alpha_max = (float)need(*c, "alpha_max").as_num();
        d.pml[a][s].beta_max = (float)need(*c, "beta_max").as_num();
        d.pml[a][s].ref_vel = (float)need(*c, "ref_vel").as_num();
      }
      if (b->get("ablexp")) fail(std::string(bnames[a][s]) + ": ablexp is not on this path (use cfspml)");
      if (const Value *f = b->get("free")) {
        if (!(a == 2 && s == 1)) fail("free surface is only implemented at the top");
        if (f->as_str() != "timg") fail("free surface type must be \"timg\"");
        d.free_top = 1;
      }
    }

  // ---- grid (main:158-199)
  std::vector<float> coord(3 * g.siz, 0.f);
  const Value &gg = need(par, "grid_generation_method");
  if (const Value *imp = gg.get("import")) {
    std::string path = imp->as_str() + "/coord_" + kFnamePart + ".nc";
    import_vars(path, g, {"x", "y", "z"}, coord.data());
  } else if (const Value *cart = gg.get("cartesian")) {  // gd_curv_gen_cart, gd_t.cu:599-634
    const Value &o = need(*cart, "origin"), &h = need(*cart, "inteval");
    for (int k = -3; k < g.nk + 3; k++)
      for (int j = -3; j < g.nj + 3; j++)
        for (int i = -3; i < g.ni + 3; i++) {
          size_t p = g.at(i, j, k);
          coord[p] = (float)(o.arr.at(0).as_num() + i * h.arr.at(0).as_num());
          coord[g.siz + p] = (float)(o.arr.at(1).as_num() + j * h.arr.at(1).as_num());
          coord[2 * g.siz + p] = (float)(o.arr.at(2).as_num() + k * h.arr.at(2).as_num());
        }
  } else {
    fail("grid_generation_method must be import or cartesian");
  }
  if (gg.get("import") && cgfd_fill_ghosts(g.ni, g.nj, g.nk, 3, coord.data())) fail(cgfd_last_error());

  // ---- metrics (main:201-228): imported here, or calculated on the GPU after the dt check
  std::vector<float> metric(10 * g.siz, 0.f);
  const Value &mm = need(par, "metric_calculation_method");
  const bool metric_import = mm.get("import") != nullptr;
  if (metric_import) {
    std::string path = mm.get("import")->as_str() + "/metric_" + kFnamePart + ".nc";
    import_vars(path, g, {"jac", "xi_x", "xi_y", "xi_z", "eta_x", "eta_y", "eta_z", "zeta_x", "zeta_y", "zeta_z"},
                metric.data());
    cgfd_fill_ghosts(g.ni, g.nj, g.nk, 10, metric.data());
  }

  // ---- medium (par_t.cu:428-721, md_import md_t.cu:269-326)
  const Value &md = need(par, "medium");
  std::string type = need(md, "type").as_str();
  std::vector<std::string> mnames;
  if (type == "acoustic_iso") {
    d.medium_type = CGFD_MEDIUM_ACOUSTIC_ISO;
    mnames = {"rho", "kappa"};
    g_ncmp = 4;
    g_names = kAcNames;
  } else if (type == "elastic_iso") { d.medium_type = CGFD_MEDIUM_ELASTIC_ISO; mnames = {"rho", "lambda", "mu"}; }
  else if (type == "elastic_vti") { d.medium_type = CGFD_MEDIUM_ELASTIC_VTI; mnames = {"rho", "c11", "c13", "c33", "c55", "c66"}; }
  else if (type == "elastic_aniso") {
    d.medium_type = CGFD_MEDIUM_ELASTIC_ANISO;
    mnames = {"rho"};
    for (int a = 1; a <= 6; a++)
      for (int b = a; b <= 6; b++) mnames.push_back("c" + std::to_string(a) + std::to_string(b));
  } else if (type == "viscoelastic_iso") {
    // generalized Maxwell body (par_t.cu:730-770; only visco_type gmb reaches the time loop)
    d.medium_type = CGFD_MEDIUM_VISCO_ISO;
    mnames = {"rho", "lambda", "mu", "Qp", "Qs"};
    const Value &vc = need(par, "visco_config");
    if (need(vc, "visco_type").as_str() != "gmb") fail("visco_type must be gmb (graves_Qs is not applied by the time loop)");
    static cgfd_visco_desc vd;
    vd.nmaxwell = need(vc, "number_of_maxwell").as_int();
    vd.fmin = (float)need(vc, "min_freq").as_num();
    vd.fmax = (float)need(vc, "max_freq").as_num();
    vd.fr = (float)need(vc, "refer_freq").as_num();
    d.visco = &vd;
  } else fail("medium type '" + type + "' is not on this path (acoustic_iso, elastic_iso/vti/aniso, viscoelastic_iso)");
  std::string way = need(md, "input_way").as_str();
  // visco-elastic Q volumes come from one-component media files (media_*2model_onecmp), not built
  if (d.medium_type == CGFD_MEDIUM_VISCO_ISO && way != "import")
    fail("viscoelastic_iso media are read with input_way 'import' (rho lambda mu Qp Qs); their one-component "
         "Qp / Qs files are not on this path");
  std::vector<float> medium(mnames.size() * g.siz, 0.f);
  if (way == "import") {
    import_vars(need(md, "import").as_str() + "/media_" + kFnamePart + ".nc", g, mnames, medium.data());
  } else if (way == "infile_layer") {
    // layer model discretised on the GPU (media_layer2model_el_iso / _el_vti / _el_aniso,
    // main_curv_col_el_3d.cu:301-336), into the medium order of the medium type
    cgfd::fmt::LayerFile lf = cgfd::fmt::read_layer_file(need(md, "infile_layer").as_str());
    const std::string em = md.get("equivalent_medium_method") ? md.get("equivalent_medium_method")->as_str() : "loc";
    const int method = em == "loc" ? CGFD_MEDIA_LOC : em == "har" ? CGFD_MEDIA_HAR : em == "ari" ? CGFD_MEDIA_ARI : -1;
    if (method < 0) fail("equivalent_medium_method '" + em + "' must be loc, har or ari");
    if (cgfd_media_layer_gpu(gpu, g.ni, g.nj, g.nk, coord.data(), &lf.media(), d.medium_type, method, medium.data()))
      fail(std::string("media on the GPU: ") + cgfd_last_error());
  } else if (way == "infile_grid") {
    // grid model discretised on the GPU (media_grid2model_el_iso / _el_vti / _el_aniso,
    // main_curv_col_el_3d.cu:365-420; the reference reads no acoustic grid files there)
    if (d.medium_type == CGFD_MEDIUM_ACOUSTIC_ISO) fail("medium input_way 'infile_grid' is read for elastic media only");
    cgfd::fmt::GridFile gf = cgfd::fmt::read_grid_file(need(md, "infile_grid").as_str());
    const std::string em = md.get("equivalent_medium_method") ? md.get("equivalent_medium_method")->as_str() : "loc";
    const int method = em == "loc" ? CGFD_MEDIA_LOC : em == "har" ? CGFD_MEDIA_HAR : em == "ari" ? CGFD_MEDIA_ARI : -1;
    if (method < 0) fail("equivalent_medium_method '" + em + "' must be loc, har or ari");
    if (cgfd_media_grid_gpu(gpu, g.ni, g.nj, g.nk, coord.data(), &gf.desc(), d.medium_type, method, medium.data()))
      fail(std::string("media on the GPU: ") + cgfd_last_error());
  } else if (way == "binfile") {
    // 3-D binary model discretised on the GPU (media_bin2model_el_iso, main_curv_col_el_3d.cu:439-458;
    // the reference reads binary models for elastic_iso media only)
    if (d.medium_type != CGFD_MEDIUM_ELASTIC_ISO) fail("medium input_way 'binfile' is read for elastic_iso media only");
    const Value &bf = need(md, "binfile");
    cgfd_bin_model bm{};
    const char *keys[3] = {"dim1", "dim2", "dim3"};
    for (int q = 0; q < 3; q++) {
      const std::string a = need(bf, keys[q]).as_str();
      bm.order[q] = a == "x" ? 0 : a == "y" ? 1 : a == "z" ? 2 : -1;
      bm.size[q] = need(bf, "size").arr.at(q).as_int();
      bm.spacing[q] = (float)need(bf, "spacing").arr.at(q).as_num();
      bm.origin[q] = (float)need(bf, "origin").arr.at(q).as_num();
    }
    const size_t nvol = (size_t)bm.size[0] * bm.size[1] * bm.size[2];
    std::vector<float> vol[3];
    const char *files[3] = {"rho", "Vp", "Vs"};
    for (int q = 0; q < 3; q++) {  // raw float32, file order (read_bin_file, media_read_file.cpp:1274-1320)
      const std::string path = need(bf, files[q]).as_str();
      FILE *fp = fopen(path.c_str(), "rb");
      if (!fp) fail("cannot open " + path);
      vol[q].resize(nvol);
      const size_t got = fread(vol[q].data(), sizeof(float), nvol, fp);
      fclose(fp);
      if (got < nvol) fail("Insufficient data in " + path);
    }
    bm.rho = vol[0].data(); bm.vp = vol[1].data(); bm.vs = vol[2].data();
    if (cgfd_media_bin_el_iso_gpu(gpu, g.ni, g.nj, g.nk, coord.data(), &bm, medium.data()))
      fail(std::string("media on the GPU: ") + cgfd_last_error());
  } else {
    fail("medium input_way '" + way + "' is not on this path (import, infile_layer, infile_grid or binfile)");
  }

  d.ni = g.ni; d.nj = g.nj; d.nk = g.nk;
  d.coord = coord.data();
  d.metric = metric.data();
  d.medium = medium.data();

  // ---- dt check in FP64 (main:591-648)
  if (check == 1) {
    double dtmax = 0.0;
    if (cgfd_dt_estimate(&d, 1.3, &dtmax)) fail(cgfd_last_error());
    printf("maximum allowed time step = %g\n", dtmax);
    if (dtmax <= 0.0) fail("maximum dt <= 0");
    if (dt < 0.0) {
      dt = cgfd_keep_three_digits(dtmax);
      nt_total = (int)(twin / dt + 0.5);  // main:621 (no +1 in this branch)
      printf("-> set dt = %g, nt_total = %d\n", dt, nt_total);
    }
    if (dtmax < dt) fail("dt = " + std::to_string(dt) + " > dtmax = " + std::to_string(dtmax));
  }
  if (dt <= 0.0) fail("no time step");
  // FP64 metrics on the GPU (equal to the host FP64 calculation bitwise)
  if (!metric_import && cgfd_metric_calc_gpu(gpu, g.ni, g.nj, g.nk, coord.data(), metric.data()))
    fail(std::string("metrics on the GPU: ") + cgfd_last_error());
  d.dt = (float)dt;
  d.t0 = (float)t0;
  d.nt_total = nt_total;

  // ---- sources and stations
  cgfd::fmt::SourceFile sf = cgfd::fmt::read_source_file(need(par, "in_source_file").as_str());
  d.src = sf.desc();
  cgfd::fmt::StationFile stf;
  bool have_sta = par.get("in_station_file") != nullptr;
  if (have_sta) {
    stf = cgfd::fmt::read_station_file(par.get("in_station_file")->as_str());
    d.sta = stf.desc();
  }
  std::string out = par.get("output_dir") ? par.get("output_dir")->as_str() : std::string(".");
  mkdirs(out);
  d.precision = CGFD_PREC_FP32;
  d.device = gpu;

  // ---- run
  cgfd_problem *p = nullptr;
  if (cgfd_problem_create(&d, &p)) fail(std::string("create: ") + cgfd_last_error());
  printf("grid %d x %d x %d, dt %g, nt_total %d, device %.2f GB\n", g.ni, g.nj, g.nk, dt, nt_total,
         cgfd_device_bytes(p) / 1e9);
  // snapshots (io_snapshot_locate + io_snap_nc_create); taken at the start of a step
  std::vector<Snap> snaps;
  if (const Value *sv = par.get("snapshot"))
    for (const Value &e : sv->arr) {
      snaps.push_back(parse_snapshot(e, g));
      open_snapshot(snaps.back(), out);
    }
  // line receivers and slices, sampled on the device at the start of every step
  std::vector<LinePoint> lines = parse_lines(par.get("receiver_line"), g);
  if (!lines.empty()) {
    std::vector<int> ijk;
    for (const LinePoint &l : lines) ijk.insert(ijk.end(), {l.i, l.j, l.k});
    if (cgfd_set_line_receivers(p, (int)lines.size(), ijk.data())) fail(std::string("lines: ") + cgfd_last_error());
  }
  Slices slices = open_slices(par.get("slice"), g, out);
  int ring = 100;  // steps per run chunk; the slice ring holds one chunk (at most ~512 MB)
  {
    const size_t per = 9 * sizeof(float) *
                       (slices.idx[0].size() * g.nk * g.nj + slices.idx[1].size() * g.nk * g.ni +
                        slices.idx[2].size() * g.nj * g.ni);
    if (per > 0) {
      ring = (int)std::max<size_t>(1, std::min<size_t>(100, (size_t(512) << 20) / per));
      if (cgfd_set_slices(p, (int)slices.idx[0].size(), slices.idx[0].data(), (int)slices.idx[1].size(),
                          slices.idx[1].data(), (int)slices.idx[2].size(), slices.idx[2].data(), ring))
        fail(std::string("slices: ") + cgfd_last_error());
    }
  }
  std::vector<float> slice_buf;
  auto next_snapshot = [&](int from) {
    int best = nt_total;
    for (const Snap &s : snaps)
      for (int it = std::max(from, s.it1); it < nt_total; it++)
        if (snapshot_due(s, it, nt_total)) { best = std::min(best, it); break; }
    return best;
  };
  int step = 0, last_print = 0;
  while (step < nt_total) {
    for (Snap &s : snaps)
      if (snapshot_due(s, step, nt_total))
        put_snapshot(s, p, g, medium, d.medium_type == CGFD_MEDIUM_ELASTIC_ISO,
                     (float)step * d.dt + d.t0);  // t_cur = it * dt + t0 in float (drv_rk_curv_col.cu:195)
    int n = std::min({ring, nt_total - step, std::max(1, next_snapshot(step + 1) - step)});
    int rc = cgfd_run(p, n);
    if (rc) { std::string m = cgfd_last_error(); cgfd_problem_destroy(p); fail("run: " + m); }
    for (int it = step; it < step + n && !slices.idx[0].empty() + !slices.idx[1].empty() + !slices.idx[2].empty(); it++)
      put_slices(slices, p, g, it, (float)it * d.dt + d.t0, slice_buf);
    step += n;
    if (step - last_print >= 100 || step == nt_total) {
      printf("-> it=%d\n", step);
      fflush(stdout);
      last_print = step;
    }
  }
  snaps.clear();  // closes the snapshot files
  for (auto &f : slices.files) f.clear();  // closes the slice files
  // line receivers (io_line_output_sac, io_funcs.cu:1943-1985): <line>.no<seq>.<cmp>.sac
  if (!lines.empty()) {
    std::vector<float> ls(lines.size() * 9 * (size_t)nt_total);
    if (cgfd_get_line_seismograms(p, ls.data())) fail(std::string("lines: ") + cgfd_last_error());
    for (size_t r = 0; r < lines.size(); r++) {
      const LinePoint &l = lines[r];
      const size_t c0 = g.at(l.i, l.j, l.k);
      for (int c = 0; c < g_ncmp; c++)
        cgfd::fmt::write_sac(out + "/" + l.line + ".no" + std::to_string(l.seq) + "." + g_names[c] + ".sac",
                             &ls[(r * 9 + c) * nt_total], nt_total, (float)dt, coord[c0], coord[g.siz + c0],
                             coord[2 * g.siz + c0], (float)dt);
    }
    printf("wrote %zu line receivers\n", lines.size());
  }

  // ---- SAC output (io_recv_output_sac, io_funcs.cu:1775-1902)
  int nsta = cgfd_num_stations(p);
  std::vector<float> seis((size_t)std::max(nsta, 0) * 9 * nt_total);
  std::vector<int> idx(std::max(nsta, 1)), ijk(3 * std::max(nsta, 1));
  if (nsta > 0) {
    cgfd_get_seismograms(p, seis.data());
    cgfd_station_info(p, idx.data(), ijk.data());
  }
  // free-surface peak ground motion (PG_slice_output, io_funcs.cu:2065-2124)
  if (d.free_top) {
    const size_t nx = g.ni + 6, ny = g.nj + 6;
    std::vector<float> pg(15 * nx * ny);
    if (cgfd_get_peak_motion(p, 0, pg.data())) fail(std::string("peak motion: ") + cgfd_last_error());
    cgfd::nc::File f;
    f.version = 1;  // NC_CLOBBER: classic format
    f.dims = {{"j", ny}, {"i", nx}};
    const char *names[15] = {"PGV", "PGVh", "PGVx", "PGVy", "PGVz", "PGA", "PGAh", "PGAx",
                             "PGAy", "PGAz", "PGD", "PGDh", "PGDx", "PGDy", "PGDz"};
    std::vector<const float *> data;
    for (int q = 0; q < 15; q++) {
      cgfd::nc::Var v;
      v.name = names[q];
      v.dimids = {0, 1};
      f.vars.push_back(v);
      data.push_back(pg.data() + (size_t)q * nx * ny);
    }
    f.gatts.push_back({"global_index_of_first_physical_points", cgfd::nc::INT, {0.0, 0.0}, ""});
    f.gatts.push_back({"count_index_of_physical_points", cgfd::nc::INT, {(double)g.ni, (double)g.nj}, ""});
    f.gatts.push_back({"coords_of_mpi_topo", cgfd::nc::INT, {0.0, 0.0, 0.0}, ""});
    cgfd::nc::write(out + "/PG_V_A_D_px0_py0_pz0.nc", f, data);
  }
  cgfd_problem_destroy(p);
  for (int r = 0; r < nsta; r++) {
    size_t c0 = g.at(ijk[3 * r], ijk[3 * r + 1], ijk[3 * r + 2]);
    float x = coord[c0], y = coord[g.siz + c0], z = coord[2 * g.siz + c0];
    const std::string &name = stf.names[idx[r]];
    float *tr = &seis[(size_t)r * 9 * nt_total];
    for (int c = 0; c < g_ncmp; c++)
      cgfd::fmt::write_sac(out + "/" + name + "." + g_names[c] + ".sac", tr + (size_t)c * nt_total, nt_total,
                           (float)dt, x, y, z, (float)dt);
    if (d.medium_type == CGFD_MEDIUM_ELASTIC_ISO) {
      // strain from stress in place (io_recv_output_sac_el_iso_strain, io_funcs.cu:1821-1902)
      float lam = medium[g.siz + c0], mu = medium[2 * g.siz + c0];
      float E1 = (float)((lam + mu) / (mu * (3.0 * lam + 2.0 * mu)));
      float E2 = (float)(-lam / (2.0 * mu * (3.0 * lam + 2.0 * mu)));
      float E3 = (float)(1.0 / mu);
      float *T[6];
      for (int c = 0; c < 6; c++) T[c] = tr + (size_t)(3 + c) * nt_total;
      for (int t = 0; t < nt_total; t++) {
        float E0 = E2 * (T[0][t] + T[1][t] + T[2][t]);
        T[0][t] = E0 - (E2 - E1) * T[0][t];
        T[1][t] = E0 - (E2 - E1) * T[1][t];
        T[2][t] = E0 - (E2 - E1) * T[2][t];
        T[3][t] = 0.5f * E3 * T[3][t];
        T[4][t] = 0.5f * E3 * T[4][t];
        T[5][t] = 0.5f * E3 * T[5][t];
      }
      const char *en[6] = {"Exx", "Eyy", "Ezz", "Eyz", "Exz", "Exy"};
      for (int c = 0; c < 6; c++)
        cgfd::fmt::write_sac(out + "/" + name + "." + en[c] + ".sac", T[c], nt_total, (float)dt, x, y, z, (float)dt);
    }
  }
  printf("wrote %d stations to %s\n", nsta, out.c_str());
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    return run(argc, argv);
  } catch (std::exception &e) {
    fprintf(stderr, "cgfd3d_b200: %s\n", e.what());
    return 1;
  }
}
