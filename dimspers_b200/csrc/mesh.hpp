// Host-side split-1 annulus mesh in the reference's numbering, plus the
// structured P2 lattice view the device kernels use.
//
// Reference numbering (src/Grid/mesher.jl):
//   vertices  node = ir + nr*itheta (0-based), theta-major        :166-172
//   quads     q = ir + (nr-1)*itheta; tris 2q = [1,2,4], 2q+1 = [2,3,4]  :174-200
//   midpoints nvert + edge id, edges numbered first-seen over (element,
//             local edge (1,2),(2,3),(3,1))                       :349-392
// Device lattice: node (a, b), a = 0..2*ncr radial, b = 0..2*nct-1 angular
// (periodic), index a + (2*ncr+1)*b.  Every reference node maps to one
// lattice node; the permutation is built from the endpoints of each edge.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dp {

struct Mesh {
  int ncr = 0, nct = 0;         // radial / angular cells
  double r_in = 1.22, r_out = 2.22;
  int pressure = 1;             // dp_pressure_space
  int64_t nel = 0, nvert = 0, nnod = 0, npres = 0, nfixed = 0;
  std::vector<int64_t> e2n;     // 6*nel, 0-based, element-major (e*6 + k)
  std::vector<double> theta, r; // nnod, reference numbering
  std::vector<int32_t> colors;  // nel, 1-based
  int32_t ncolors = 0;
  std::vector<int64_t> ref2lat; // nnod
  std::vector<int64_t> lat2ref; // nnod
  std::vector<int64_t> omega;   // fixed DOFs, 0-based (2*node+1), top then bottom

  int64_t A() const { return 2 * (int64_t)ncr + 1; }  // nodes per radial line
  int64_t B() const { return 2 * (int64_t)nct; }      // angular lattice size
};

// Validates the description; returns an empty string on success.
std::string check_desc(int ncr, int nct, double r_in, double r_out, int pressure);

void mesh_sizes(int ncr, int nct, int pressure, int64_t* nel, int64_t* nnod, int64_t* npres,
                int64_t* nfixed);

// Builds everything above.  with_colors=false skips the greedy colouring.
void build_mesh(Mesh& m, int ncr, int nct, double r_in, double r_out, int pressure,
                bool with_colors = true);

}  // namespace dp
