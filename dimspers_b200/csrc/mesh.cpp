// Host-side split-1 annulus mesh: vertices, split-1 triangles, first-seen edge
// (midpoint) numbering, seam-aware midpoint coordinates, greedy colouring,
// free-slip set and the reference <-> lattice permutation.
//
// Reference: src/Grid/mesher.jl:152-233 (Grid_split1), :313-347
// (element_neighbours), :349-392 (edge_connectivity), :394-417
// (add_midpoints), :419-441 (point_ids); src/Grid/coloring.jl:5-64
// (color_mesh); src/Setup/boundary_conditions.jl:15-37 (free_slip).
//
// edge_connectivity hands out a new id only when (element, local edge) meets
// an edge no earlier element contains, so its ids are the first-seen order of
// the edges; this file reproduces that order with a per-vertex edge table
// instead of the reference's neighbour search.  color_mesh is greedy
// first-fit over vertex-sharing elements in element order; the colour set of
// the neighbours does not depend on the order they are visited in.
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace dp {

std::string check_desc(int ncr, int nct, double r_in, double r_out, int pressure) {
  if (ncr < 1) return "nr_cells must be >= 1";
  if (nct < 3) return "ntheta_cells must be >= 3";
  if (!(r_in > 0.0) || !(r_out > r_in)) return "radii must satisfy 0 < r_in < r_out";
  if (pressure != 0 && pressure != 1) return "pressure_space must be 0 (continuous) or 1 (discontinuous)";
  if ((int64_t)ncr * (int64_t)nct > (int64_t)1 << 28) return "mesh too large";
  return std::string();
}

void mesh_sizes(int ncr, int nct, int pressure, int64_t* nel, int64_t* nnod, int64_t* npres,
                int64_t* nfixed) {
  const int64_t ne = 2 * (int64_t)ncr * nct;
  const int64_t nv = (int64_t)(ncr + 1) * nct;
  if (nel) *nel = ne;
  if (nnod) *nnod = (2 * (int64_t)ncr + 1) * 2 * (int64_t)nct;
  if (npres) *npres = pressure == 0 ? nv : 3 * ne;
  if (nfixed) *nfixed = 2 * 2 * (int64_t)nct;
}

void build_mesh(Mesh& m, int ncr, int nct, double r_in, double r_out, int pressure,
                bool with_colors) {
  m.ncr = ncr;
  m.nct = nct;
  m.r_in = r_in;
  m.r_out = r_out;
  m.pressure = pressure;
  const int nr = ncr + 1;            // radial nodes as in the reference
  const int64_t nv = (int64_t)nr * nct;
  m.nvert = nv;
  mesh_sizes(ncr, nct, pressure, &m.nel, &m.nnod, &m.npres, &m.nfixed);
  const int64_t nel = m.nel;

  // -- vertices (mesher.jl:166-172): LinRange element (1-t)*a + t*b, t = j/(n-1)
  m.theta.assign(m.nnod, 0.0);
  m.r.assign(m.nnod, 0.0);
  const double two_pi = 2.0 * 3.14159265358979323846;
  const double dth = two_pi / (double)nct;
  for (int it = 0; it < nct; ++it)
    for (int ir = 0; ir < nr; ++ir) {
      const int64_t n = ir + (int64_t)nr * it;
      const double t = (double)ir / (double)(nr - 1);
      m.r[n] = (1.0 - t) * r_in + t * r_out;
      m.theta[n] = 0.0 + (dth * (double)it) * 1.0;
    }

  // -- split-1 triangles (mesher.jl:174-200)
  m.e2n.assign(6 * nel, 0);
  for (int it = 0; it < nct; ++it)
    for (int ir = 0; ir < ncr; ++ir) {
      const int64_t q = ir + (int64_t)ncr * it;
      const int64_t i1 = ir + (int64_t)nr * it;
      const int64_t i2 = (it < nct - 1) ? ir + (int64_t)nr * (it + 1) : (int64_t)ir;
      const int64_t v[4] = {i1, i2, i2 + 1, i1 + 1};
      int64_t* a = &m.e2n[6 * (2 * q)];
      int64_t* b = &m.e2n[6 * (2 * q + 1)];
      a[0] = v[0]; a[1] = v[1]; a[2] = v[3];
      b[0] = v[1]; b[1] = v[2]; b[2] = v[3];
    }

  // -- first-seen edge numbering (mesher.jl:349-392)
  const int kSlots = 8;  // a vertex of this mesh has at most 6 incident edges
  std::vector<int64_t> slot_other(nv * kSlots, -1), slot_id(nv * kSlots, -1);
  std::vector<int64_t> edge_lo, edge_hi;
  edge_lo.reserve(3 * nel / 2 + nct);
  edge_hi.reserve(3 * nel / 2 + nct);
  static const int lm[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  for (int64_t e = 0; e < nel; ++e) {
    int64_t* en = &m.e2n[6 * e];
    for (int k = 0; k < 3; ++k) {
      int64_t lo = en[lm[k][0]], hi = en[lm[k][1]];
      if (lo > hi) std::swap(lo, hi);
      int64_t id = -1;
      int s = 0;
      for (; s < kSlots; ++s) {
        const int64_t o = slot_other[lo * kSlots + s];
        if (o == hi) { id = slot_id[lo * kSlots + s]; break; }
        if (o < 0) break;
      }
      if (id < 0) {
        if (s >= kSlots) throw std::runtime_error("vertex edge table overflow");
        id = (int64_t)edge_lo.size();
        slot_other[lo * kSlots + s] = hi;
        slot_id[lo * kSlots + s] = id;
        edge_lo.push_back(lo);
        edge_hi.push_back(hi);
      }
      en[3 + k] = nv + id;
    }
  }
  if (nv + (int64_t)edge_lo.size() != m.nnod) throw std::runtime_error("unexpected node count");

  // -- midpoint coordinates (mesher.jl:394-417)
  for (size_t i = 0; i < edge_lo.size(); ++i) {
    double t1 = m.theta[edge_lo[i]], t2 = m.theta[edge_hi[i]];
    if (std::fabs(t1 - t2) > 3.14159265358979323846) {
      if (t1 < 3.14159265358979323846) t1 += two_pi;
      if (t2 < 3.14159265358979323846) t2 += two_pi;
    }
    m.theta[nv + i] = 0.5 * (t1 + t2);
    m.r[nv + i] = 0.5 * (m.r[edge_lo[i]] + m.r[edge_hi[i]]);
  }

  // -- reference <-> lattice permutation
  const int64_t A = m.A(), B = m.B();
  m.ref2lat.assign(m.nnod, -1);
  m.lat2ref.assign(m.nnod, -1);
  auto vlat_a = [&](int64_t v) { return 2 * (v % nr); };
  auto vlat_b = [&](int64_t v) { return 2 * (v / nr); };
  for (int64_t v = 0; v < nv; ++v) m.ref2lat[v] = vlat_a(v) + A * vlat_b(v);
  for (size_t i = 0; i < edge_lo.size(); ++i) {
    const int64_t a = (vlat_a(edge_lo[i]) + vlat_a(edge_hi[i])) / 2;
    int64_t b1 = vlat_b(edge_lo[i]), b2 = vlat_b(edge_hi[i]);
    if (std::llabs(b1 - b2) > 2) {  // seam edge: unwrap the b = 0 end
      if (b1 < b2) b1 += B; else b2 += B;
    }
    const int64_t b = ((b1 + b2) / 2) % B;
    m.ref2lat[nv + i] = a + A * b;
  }
  for (int64_t n = 0; n < m.nnod; ++n) {
    const int64_t l = m.ref2lat[n];
    if (l < 0 || l >= m.nnod || m.lat2ref[l] >= 0) throw std::runtime_error("lattice permutation is not a bijection");
    m.lat2ref[l] = n;
  }

  // -- free slip (boundary_conditions.jl:27-37): top (r == rmax) then bottom
  double rmin = m.r[0], rmax = m.r[0];
  for (int64_t n = 0; n < m.nnod; ++n) { rmin = std::min(rmin, m.r[n]); rmax = std::max(rmax, m.r[n]); }
  m.omega.clear();
  for (int64_t n = 0; n < m.nnod; ++n) if (m.r[n] == rmax) m.omega.push_back(2 * n + 1);
  for (int64_t n = 0; n < m.nnod; ++n) if (m.r[n] == rmin) m.omega.push_back(2 * n + 1);

  // -- greedy colouring (coloring.jl:5-64)
  m.colors.assign(nel, 0);
  m.ncolors = 0;
  if (!with_colors) return;
  std::vector<int64_t> vstart(nv + 1, 0), vlist(3 * nel);
  for (int64_t e = 0; e < nel; ++e)
    for (int k = 0; k < 3; ++k) vstart[m.e2n[6 * e + k] + 1]++;
  for (int64_t v = 0; v < nv; ++v) vstart[v + 1] += vstart[v];
  std::vector<int64_t> fill(vstart.begin(), vstart.end() - 1);
  for (int64_t e = 0; e < nel; ++e)
    for (int k = 0; k < 3; ++k) vlist[fill[m.e2n[6 * e + k]]++] = e;
  std::vector<uint8_t> used;
  for (int64_t e = 0; e < nel; ++e) {
    used.assign(m.ncolors + 2, 0);
    for (int k = 0; k < 3; ++k) {
      const int64_t v = m.e2n[6 * e + k];
      for (int64_t j = vstart[v]; j < vstart[v + 1]; ++j) {
        const int64_t o = vlist[j];
        if (o != e && m.colors[o] != 0) used[m.colors[o]] = 1;
      }
    }
    int c = 1;
    while (c <= m.ncolors && used[c]) ++c;
    if (c > m.ncolors) m.ncolors = c;
    m.colors[e] = c;
  }
}

}  // namespace dp
