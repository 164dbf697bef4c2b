// The reference-side driver a maintainer adds beside main/gpu_offload.cpp:
// DATA.json through the reference's own DATA struct (main/mpm_data.h), the
// time loop on libdampm_cuda through the C ABI of include/dampm_cuda.h.
// Built by `make binding` in oracle/ (it needs the reference checkout for
// mpm_data.h); tests/test_gpu_binding.py runs it and compares its output
// with the Python binding's.
//
// Output: the loop state on stdout ("it=<it> t=<t> np=<np>") and, in
// state.bin, np doubles each of x, y, vpx, vpy, hp in reference order.
#include <cstdio>
#include <cstdlib>
#include <fstream>  // mpm_data.h reads DATA.json with std::ifstream
#include <string>
#include <vector>

#include "mpm_data.h"
#include "dampm_cuda.h"

static void check(dampm_ctx* c, int rc) {
  if (rc) {
    std::fprintf(stderr, "dampm: %d %s\n", rc, c ? dampm_last_error(c) : "");
    std::exit(1);
  }
}

int main() {
  DATA d("DATA.json");
  dampm_grid g{d.Nex, d.Ney, d.hx, d.hy};
  dampm_params p{d.g, d.T, d.rho, d.xi, d.mu, d.phi, d.tauy, d.BINGHAM_ON,
                 d.FRICTION_ON, d.CFL, d.BC_FLAG, d.MERGE_SPLIT_ON, d.eq_level,
                 d.DT_FIXED, d.NSTEPS};
  dampm_ms_params m{d.ms_alpha, d.ms_beta, d.ms_split_hp_min, d.ms_shear_split,
                    d.ms_hp_min, d.ms_max_dv, d.ms_min_level, d.ms_max_level,
                    d.ms_min_particles_per_cell, d.ms_call_interval, d.ms_max_ops};
  dampm_ctx* c = nullptr;
  check(c, dampm_ctx_create(&g, &p, &m, DAMPM_FP64, /*capacity*/ 0, /*stream*/ nullptr, &c));
  check(c, dampm_upload_terrain(c, d.Z.data(), d.dZdx.data(), d.dZdy.data()));
  check(c, dampm_upload_particles(c, (long long)d.x.size(), d.x.data(), d.y.data(),
                                  d.Mp.data(), d.Ap.data(), d.vpx.data(), d.vpy.data(),
                                  d.hp.data(), d.mom_px.data(), d.mom_py.data(), d.Vp.data()));
  check(c, dampm_enable_merge_split(c, d.MERGE_SPLIT_ON));  // gpu_offload cadence
  long long done = 0;
  check(c, dampm_run(c, /*max_steps*/ 1LL << 40, /*chunk*/ 256, &done));
  int it = 0;
  double t = 0, dt = 0;
  long long np = 0;
  check(c, dampm_status(c, &it, &t, &dt, &np));
  std::FILE* f = std::fopen("state.bin", "wb");
  if (!f) return 1;
  std::vector<double> buf(np > 0 ? np : 1);
  for (const char* name : {"x", "y", "vpx", "vpy", "hp"}) {
    check(c, dampm_download(c, name, buf.data()));
    std::fwrite(buf.data(), sizeof(double), size_t(np), f);
  }
  std::fclose(f);
  std::printf("it=%d t=%.17g np=%lld\n", it, t, np);
  dampm_ctx_destroy(c);
  return 0;
}
