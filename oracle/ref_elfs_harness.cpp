// TEST INFRASTRUCTURE ONLY -- runs the reference's own ELFS
// adaptive_merge_split (main/merge_split_ops.h:720-755, compiled unmodified
// against the stand-in headers in ref_shim/) on a particle state read from a
// binary file, and writes the result.
//
// input  (little-endian): int32 Nex, Ney; f64 hx, hy; 5 f64 ms_config values
//   (alpha, beta, hp_min, max_dv, stretch_thresh); int32 min_level,
//   max_level, call_interval; f64 max_ops; int32 np; int32 nd; then nd times
//   { int32 name_len; name; f64[np] }; then x[np], y[np]; then level
//   int32[np], label int32[np]
// output: int32 np_new; then the dprops in map order {name, f64[np_new]},
//   x, y, level, label.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "merge_split_ops.h"

template <class T>
static void rd(std::ifstream& f, T& v) { f.read(reinterpret_cast<char*>(&v), sizeof v); }
template <class T>
static void rdv(std::ifstream& f, std::vector<T>& v, size_t n) {
  v.resize(n);
  f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
}
template <class T>
static void wr(std::ofstream& f, const T& v) { f.write(reinterpret_cast<const char*>(&v), sizeof v); }

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  std::ifstream f(argv[1], std::ios::binary);
  int32_t Nex, Ney;
  double hx, hy;
  rd(f, Nex); rd(f, Ney); rd(f, hx); rd(f, hy);
  ms_config cfg;
  rd(f, cfg.alpha); rd(f, cfg.beta); rd(f, cfg.hp_min); rd(f, cfg.max_dv);
  rd(f, cfg.stretch_thresh);
  int32_t a, b, c;
  rd(f, a); rd(f, b); rd(f, c);
  cfg.min_level = a; cfg.max_level = b; cfg.call_interval = c;
  double max_ops;
  rd(f, max_ops);
  cfg.max_ops = (int)max_ops;
  int32_t np, nd;
  rd(f, np); rd(f, nd);
  std::vector<std::string> names;
  std::vector<std::vector<double>> cols;
  for (int k = 0; k < nd; ++k) {
    int32_t len;
    rd(f, len);
    std::string s(len, ' ');
    f.read(&s[0], len);
    names.push_back(s);
    std::vector<double> v;
    rdv(f, v, np);
    cols.push_back(v);
  }
  std::vector<double> x, y;
  rdv(f, x, np);
  rdv(f, y, np);
  std::vector<int32_t> level, label;
  rdv(f, level, np);
  rdv(f, label, np);

  quadgrid_t<std::vector<double>> grid;
  grid.set_sizes(Ney, Nex, hx, hy);
  particles_t ptcls(np, {"label", "level"}, names, grid, x, y);
  for (int k = 0; k < nd; ++k) ptcls.dprops[names[k]] = cols[k];
  for (int i = 0; i < np; ++i) {
    ptcls.iprops["level"][i] = level[i];
    ptcls.iprops["label"][i] = label[i];
  }
  ptcls.init_particle_mesh();
  adaptive_merge_split<particles_t::idx_t>(ptcls, cfg);

  std::ofstream o(argv[2], std::ios::binary);
  const int32_t nn = ptcls.num_particles;
  wr(o, nn);
  for (auto const& kv : ptcls.dprops) {
    const int32_t len = int32_t(kv.first.size());
    wr(o, len);
    o.write(kv.first.data(), len);
    o.write(reinterpret_cast<const char*>(kv.second.data()), sizeof(double) * nn);
  }
  o.write(reinterpret_cast<const char*>(ptcls.x.data()), sizeof(double) * nn);
  o.write(reinterpret_cast<const char*>(ptcls.y.data()), sizeof(double) * nn);
  std::vector<int32_t> lv(ptcls.iprops["level"].begin(), ptcls.iprops["level"].end());
  std::vector<int32_t> lb(ptcls.iprops["label"].begin(), ptcls.iprops["label"].end());
  o.write(reinterpret_cast<const char*>(lv.data()), sizeof(int32_t) * nn);
  o.write(reinterpret_cast<const char*>(lb.data()), sizeof(int32_t) * nn);
  return 0;
}
