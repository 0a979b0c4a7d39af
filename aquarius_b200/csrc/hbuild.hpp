// Device-side assembly of H from a three-index factor (see hbuild.cpp).
#pragma once
#include "engine.hpp"

namespace ccsd {
// the 13 spin-orbital blocks of H (2eoperator.cxx:13-21), zero-filled
void create_hamiltonian_tensors(Context& ctx, bool pack_vvvv, ccsd_hamiltonian* H);
void build_hamiltonian(Context& ctx, int naux, const double* B, const double* eps, const int* aux_per_irrep,
                       bool pack_vvvv, ccsd_hamiltonian* H);
}
