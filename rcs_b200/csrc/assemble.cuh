// Entry-assembly interface used by the C ABI and the solver.
#pragma once
#include <vector>

#include "geometry.cuh"

namespace aifmm {

// One dense tile K(rows[a], cols[b]) -> out (column-major, leading dim ld).
struct GatherBlock {
  const int* rows;
  const int* cols;
  void* out;
  int nr, nc, ld, pad;
};

struct KernelGeom {
  bool efie = true;
  int N = 0;
  EfieGeom ge{};
  EsGeom gs{};
};

struct EfieHostTables {
  std::vector<double> tri, node, len, side, locations;
  std::vector<int> rwg, edge;
};

// EFIE tables of a mesh, built on the GPU (mesh_build.cu): triangle geometry,
// and the RWG numbering of the reference's std::map over edge keys
// (src/EFIEMatrix.cpp:129-209) from a stable radix sort of the 3 nt edge keys.
void build_efie_tables_gpu(aifmm_ctx* ctx, const double* xyz, int nv, const int* tris, int nt, EfieHostTables& h);
// Octree binning on the GPU (T:576-625): the point indices in leaf order
// (stable: index order inside a leaf) and leafStart[k]..leafStart[k+1] of
// leaf k; centers = every box centre of levels 0..nLevels-1, level by level.
std::vector<int> bin_points_gpu(aifmm_ctx* ctx, const std::vector<double>& pts, const std::vector<double>& centers,
                                int nLevels, std::vector<int>& leafStart);
void build_es_tables(const double* xyz, int nv, const int* tris, int nt, std::vector<double>& tri,
                     std::vector<double>& locations);

// precision: 0 = complex128 out, 1 = complex64 out.
void launch_gather(const KernelGeom& k, const int* rows, int nr, const int* cols, int nc, int precision, void* out,
                   int ld, cudaStream_t s);
void launch_batched_gather(const KernelGeom& k, const GatherBlock* blocks_dev, const long* start_dev, int nblocks,
                           long total, int precision, cudaStream_t s);
void launch_rhs_reference(const KernelGeom& k, const double* einc, zd* out, cudaStream_t s);
void launch_rhs_plane(const KernelGeom& k, const double* khat, const double* e0, zd* out, cudaStream_t s);

}  // namespace aifmm
