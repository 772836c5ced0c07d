// Bond parameters of the C ABI (include/p3mx.h p3mx_bond_params) checked and
// converted to the device form (bonds.cuh BondParam); shared by the single-
// system and batched entry points.
#pragma once

#include "../../include/p3mx.h"
#include "bonds.cuh"
#include "common.cuh"

#include <string>
#include <vector>

namespace p3mx {

inline std::vector<BondParam> bond_types_from_abi(int n_types, const p3mx_bond_params *types,
                                                  size_t n_bonds, const int *bonds) {
  if (n_types < 0 || (n_types > 0 && !types) || (n_bonds > 0 && !bonds))
    throw Error(P3MX_EDOMAIN, "bond arrays missing");
  std::vector<BondParam> t(static_cast<size_t>(n_types));
  for (int k = 0; k < n_types; ++k) {
    auto const &s = types[k];
    if (s.kind != P3MX_BOND_FENE && s.kind != P3MX_BOND_HARMONIC)
      throw Error(P3MX_EDOMAIN, "unknown bond kind " + std::to_string(s.kind));
    if (s.kind == P3MX_BOND_FENE && !(s.r_max > 0.))
      throw Error(P3MX_EDOMAIN, "FENE parameter 'd_r_max' has to be > 0");
    if (s.r_max < 0. || s.r0 < 0.)
      throw Error(P3MX_EDOMAIN, "bond lengths have to be >= 0");
    t[k] = BondParam{s.kind == P3MX_BOND_FENE ? kBondFene : kBondHarmonic, s.k, s.r0, s.r_max};
  }
  for (size_t b = 0; b < n_bonds; ++b)
    if (bonds[3 * b] < 0 || bonds[3 * b] >= n_types)
      throw Error(P3MX_EDOMAIN, "bond type " + std::to_string(bonds[3 * b]) + " is not defined");
  return t;
}

} // namespace p3mx
