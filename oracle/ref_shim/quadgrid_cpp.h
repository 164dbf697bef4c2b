// TEST INFRASTRUCTURE ONLY -- stand-in for the grid class of the absent
// `quadgrid` submodule (.gitmodules:1-4 of the reference project,
// lucadiprofio fork, no pinned commit), restating the interface the
// reference's main/*.cpp use: set_sizes, sizes, the cell sweep with e()/gt(),
// and vtk_export.  Conventions (main/gpu_kernels.cpp:7-19): rows = Ney,
// cell id r + c*nrows, node id r + c*(nrows+1); local nodes 0 (r,c),
// 1 (r+1,c), 2 (r,c+1), 3 (r+1,c+1).  e(0)/e(1): bottom/top row,
// e(2)/e(3): left/right column.
#pragma once
#include <charconv>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

template <class T>
class quadgrid_t {
 public:
  using idx_t = int;

  void set_sizes(idx_t nr, idx_t nc, double hx, double hy) {
    nrows_ = nr;
    ncols_ = nc;
    hx_ = hx;
    hy_ = hy;
  }
  idx_t num_rows() const { return nrows_; }
  idx_t num_cols() const { return ncols_; }
  double hx() const { return hx_; }
  double hy() const { return hy_; }
  idx_t num_global_nodes() const { return (nrows_ + 1) * (ncols_ + 1); }
  idx_t num_cells() const { return nrows_ * ncols_; }

  struct cell_t {
    const quadgrid_t* g;
    idx_t id;
    idx_t r() const { return id % g->nrows_; }
    idx_t c() const { return id / g->nrows_; }
    idx_t e(idx_t k) const {
      switch (k) {
        case 0: return r() == 0 ? 0 : -1;
        case 1: return r() == g->nrows_ - 1 ? 1 : -1;
        case 2: return c() == 0 ? 2 : -1;
        case 3: return c() == g->ncols_ - 1 ? 3 : -1;
        default: return -1;
      }
    }
    idx_t gt(idx_t inode) const {
      const idx_t bl = r() + c() * (g->nrows_ + 1);
      switch (inode) {
        case 0: return bl;
        case 1: return bl + 1;
        case 2: return bl + (g->nrows_ + 1);
        default: return bl + (g->nrows_ + 2);
      }
    }
  };

  class cell_iterator {
   public:
    cell_iterator(const quadgrid_t* g, idx_t id) : c_{g, id} {}
    const cell_t* operator->() const { return &c_; }
    const cell_t& operator*() const { return c_; }
    cell_iterator& operator++() {
      ++c_.id;
      return *this;
    }
    bool operator!=(const cell_iterator& o) const { return c_.id != o.c_.id; }
    bool operator==(const cell_iterator& o) const { return c_.id == o.c_.id; }

   private:
    cell_t c_;
  };

  cell_iterator begin_cell_sweep() const { return cell_iterator(this, 0); }
  cell_iterator end_cell_sweep() const { return cell_iterator(this, num_cells()); }

  // VTK XML StructuredGrid, ASCII, points in VTK order (x fastest).
  void vtk_export(const char* filename,
                  const std::map<std::string, std::vector<double>>& vars) const {
    FILE* f = std::fopen(filename, "w");
    if (!f) return;
    const idx_t NR = nrows_ + 1, NC = ncols_ + 1;
    std::fprintf(f,
                 "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" "
                 "version=\"0.1\" byte_order=\"LittleEndian\">\n"
                 "<StructuredGrid WholeExtent=\"0 %d 0 %d 0 0\">\n<Piece Extent=\"0 %d 0 %d 0 0\">\n"
                 "<PointData>\n",
                 ncols_, nrows_, ncols_, nrows_);
    char buf[64];
    for (auto const& kv : vars) {
      std::fprintf(f, "<DataArray type=\"Float64\" Name=\"%s\" format=\"ascii\">\n", kv.first.c_str());
      for (idx_t r = 0; r < NR; ++r)
        for (idx_t c = 0; c < NC; ++c) {
          auto res = std::to_chars(buf, buf + sizeof buf, kv.second[r + c * NR]);
          *res.ptr = '\n';
          std::fwrite(buf, 1, res.ptr - buf + 1, f);
        }
      std::fprintf(f, "</DataArray>\n");
    }
    std::fprintf(f, "</PointData>\n<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (idx_t r = 0; r < NR; ++r)
      for (idx_t c = 0; c < NC; ++c) std::fprintf(f, "%.17g %.17g 0\n", c * hx_, r * hy_);
    std::fprintf(f, "</DataArray>\n</Points>\n</Piece>\n</StructuredGrid>\n</VTKFile>\n");
    std::fclose(f);
  }

 private:
  idx_t nrows_ = 0, ncols_ = 0;
  double hx_ = 1.0, hy_ = 1.0;
};
