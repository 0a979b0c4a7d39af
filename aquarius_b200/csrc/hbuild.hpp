// Device-side assembly of H from a three-index factor (see hbuild.cpp).
#pragma once
#include "engine.hpp"

namespace ccsd {
void build_hamiltonian(Context& ctx, int naux, const double* B, const double* eps, const int* aux_per_irrep,
                       bool pack_vvvv, ccsd_hamiltonian* H);
}
