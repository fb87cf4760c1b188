// Near-field K entries of RWG pairs that share a triangle, with the
// reference's own host arithmetic (near_same_triangle.cpp).
#pragma once
#include <vector>

#include "host.hpp"

namespace mlfma {

// The near-field pairs (target, source) whose RWGs share a triangle, with
// their positions in the plan's near-field order (per leaf box b, target-major
// blocks of near_sptr[b+1] - near_sptr[b] sources starting at near_zoff[b]).
void same_triangle_pairs(const Rwg& r, const Tree& t, const std::vector<int>& near_sptr,
                         const std::vector<int>& near_src, const std::vector<long long>& near_zoff,
                         std::vector<long long>& pos, std::vector<int>& tgt, std::vector<int>& src);

// z12 = -(K(k1) + K(k2)) of each pair (Code/Zmartix.h:605-612), evaluated as
// the reference does, on all host cores.
void same_triangle_z12(const Mesh& m, const Rwg& r, const Quad& q, cplx k1, cplx k2, const std::vector<int>& tgt,
                       const std::vector<int>& src, std::vector<cplx>& z12);

}  // namespace mlfma
