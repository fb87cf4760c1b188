// Host-side setup of the PMCHWT MLFMA operator: mesh, RWG numbering,
// octree, angular grids, interpolation tables and the special functions the
// transfer factors need. Everything here reproduces the reference's
// discretisation (file:line of CCCCl0uD/MLFMA_PMCHWT cited per function) so
// that the device operator matches the reference's matvec on the same mesh.
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace mlfma {

using cplx = std::complex<double>;

constexpr double kPi = 3.14159265358979323846;   // Code/PhyConstant.h:7
constexpr double kC0 = 299792458.0;              // Code/PhyConstant.h:9
constexpr double kEps0 = 2.2204e-16;             // Code/PhyConstant.h:13 (singularity threshold)
constexpr double kEta0 = 119.9169832 * kPi;      // Code/EMSource.h:78

// Triangle mesh. Point / face indices are 0-based positions in file order;
// ids are the NAS GRID / CTRIA3 numbers.
struct Mesh {
  std::vector<int> point_id;
  std::vector<double> xyz;       // [3 * points]
  std::vector<int> face_id;
  std::vector<int> face_v;       // [3 * faces] point indices
  std::vector<double> area;      // Code/NASReader.cpp:24-37
  std::vector<double> normal;    // [3 * faces], Code/NASReader.cpp:39-58 (|n_i| < 1e-6 -> 0)
};

bool read_nas(const std::string& path, Mesh& m, std::string& err);
bool mesh_from_arrays(int np, const int* pid, const double* xyz, int nf, const int* fid,
                      const int* fpts, Mesh& m, std::string& err);
void mesh_derive(Mesh& m);

// RWG functions in the reference's numbering (Code/RWGGenerator.cpp:39-113).
struct Rwg {
  int N = 0;
  std::vector<int> fpos, fneg;            // face indices of T+ / T-
  std::vector<int> free_pos, free_neg;    // point indices of the free vertices
  std::vector<int> ea, eb;                // point indices of the common edge (min id, max id)
  std::vector<double> len;                // edge length
  std::vector<double> mid;                // [3 * N] edge midpoint
};
bool build_rwgs(const Mesh& m, Rwg& r, std::string& err);

// One octree level, boxes sorted by Morton code.
struct Level {
  int level = 0;
  double len = 0.0;                       // box edge
  std::vector<uint64_t> code;
  std::vector<int> ix, iy, iz;
  std::vector<double> center;             // [3 * B]
  std::vector<int> parent;                // box index on level-1 (-1 at level 0)
  std::vector<int> child_begin;           // [B + 1] range on level+1 (children are contiguous)
  std::vector<int> near_ptr, near_idx;    // 26-neighbourhood (Code/OCTree.cpp:385-426)
  std::vector<int> far_ptr, far_idx;      // interaction list (Code/OCTree.cpp:428-488)
  std::vector<int> far_off;               // encoded offset target - source: (dx+3)*49+(dy+3)*7+(dz+3)
  int size() const { return static_cast<int>(code.size()); }
};

struct Tree {
  int maxLevel = 0;
  double leafLen = 0.0, rootLen = 0.0;
  double gmin[3] = {0, 0, 0};
  std::vector<Level> lv;                  // index = physical level 0..maxLevel
  std::vector<int> rwg_leaf;              // leaf box of each RWG
  std::vector<int> leaf_ptr, leaf_rwg;    // per leaf box: RWG ids, ascending
};
void build_tree(const Rwg& r, double leaf_target, Tree& t);

inline int encode_offset(int dx, int dy, int dz) { return (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3); }
inline void decode_offset(int e, int& dx, int& dy, int& dz) {
  dx = e / 49 - 3;
  dy = (e / 7) % 7 - 3;
  dz = e % 7 - 3;
}

// Angular grid of one level (Code/AlgoMLFMM.h:21-138): theta = acos of
// Gauss-Legendre nodes (ascending), phi_j = (j + 1/2) pi / L, j < 2L.
struct Grid {
  int L = 0, nth = 0, nph = 0, K = 0;
  std::vector<double> theta, phi, wth;    // wth: GL weights as indexed by the reference
  double wph = 0.0;                       // pi / L
  std::vector<double> khat;               // [3 * K], theta-major
};
Grid build_grid(double kabs, double box_len);

// Child-grid -> parent-grid interpolation (Code/AlgoMLFMM.h:141-189, 298-368):
// separable 3-point Lagrange in theta and in phi with periodic neighbours.
struct Interp {
  std::vector<int> tidx;   std::vector<double> lt;   // [Tp][3]
  std::vector<int> pidx;   std::vector<double> lp;   // [Pp][3]
};
Interp build_interp(const Grid& parent, const Grid& child);

// Special functions (Boost.Math's legendre_p / legendre_p_prime /
// sph_bessel / sph_neumann in the reference, Code/OverloadAlgo.h:259,
// Code/Bessel.h:14-47), from their standard recurrences.
double legendre_p(int l, double x);
double legendre_dp(int l, double x);
double sph_j(int n, double x);
double sph_y(int n, double x);
void hankel2_array(int L, double x, std::vector<cplx>& h2);
// h2_l(z), l = 0..L, for complex z by the upward recurrence from
// h2_0 = i e^{-iz}/z and h2_1 = e^{-iz} (i/z^2 - 1/z).
void hankel2_array_complex(int L, cplx z, std::vector<cplx>& h2);
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

// Triangle quadrature (Code/GaussPoints.cpp, Dunavant rules, weights sum to 1/2).
struct Quad {
  int n = 0;
  const double *l1 = nullptr, *l2 = nullptr, *l3 = nullptr, *w = nullptr;
};
bool quad_rule(int n, Quad& q);

}  // namespace mlfma
