// Device-side assembly of H from a three-index factor or dense integrals (hbuild.cpp),
// and the FCIDUMP reader (fcidump.cpp).
#pragma once
#include "engine.hpp"

namespace ccsd {
// the 13 spin-orbital blocks of H (2eoperator.cxx:13-21), zero-filled
void create_hamiltonian_tensors(Context& ctx, bool pack_vvvv, ccsd_hamiltonian* H);
void build_hamiltonian(Context& ctx, int naux, const double* B, const double* eps, const int* aux_per_irrep,
                       bool pack_vvvv, ccsd_hamiltonian* H);
// closed shell: fock[n*n] (row = upper index) and dense eri[n^4] = (pq|rs), last index
// fastest, orbitals ordered occupied first, irrep-major inside occ and vrt
void build_hamiltonian_dense(Context& ctx, int n, const double* fock, const double* eri, bool pack_vvvv,
                             ccsd_hamiltonian* H);
// the 10 plain spatial blocks of the closed-shell (RHF) Hamiltonian, zero-filled, and
// their builders from the factor / the dense integrals (arguments as above)
void create_rhf_hamiltonian_tensors(Context& ctx, ccsd_rhf_hamiltonian* H);
void build_rhf_hamiltonian(Context& ctx, int naux, const double* B, const double* eps, const int* aux_per_irrep,
                           ccsd_rhf_hamiltonian* H);
void build_rhf_hamiltonian_dense(Context& ctx, int n, const double* fock, const double* eri, ccsd_rhf_hamiltonian* H);
// the same from a (pq|rs) array already on the device (host Fock matrix)
void build_hamiltonian_device(Context& ctx, int n, const double* fock, const double* d_eri, bool pack_vvvv,
                              ccsd_hamiltonian* H);
void build_rhf_hamiltonian_device(Context& ctx, int n, const double* fock, const double* d_eri,
                                  ccsd_rhf_hamiltonian* H);
// AO -> MO on the device for a closed-shell reference: d_mo[p,q,r,s] = (pq|rs) over the
// nmo columns of C (nao x nmo, row-major), the MO Fock matrix f = C^T h C + sum_i 2(pq|ii)
// - (pi|iq) over the first nocc orbitals (host, nmo x nmo); returns sum_i (h_ii + f_ii)
double ao_to_mo(Context& ctx, int nao, int nmo, int nocc, const double* hcore, const double* eri_ao,
                const double* C, double* d_mo, double* fock);

// FCIDUMP contents: h[n*n], eri[n^4] dense, core energy
struct Fcidump {
    int norb = 0, nelec = 0;
    double ecore = 0.0;
    std::vector<double> h, eri;
};
Fcidump read_fcidump(const char* path, bool full_fock, bool header_only);
// closed-shell Fock f = h + sum_i 2(pq|ii) - (pi|iq) over the first nocc orbitals;
// returns the electronic SCF energy sum_i (h_ii + f_ii)
double closed_shell_fock(int n, int nocc, const double* h, const double* eri, double* fock);
// rotate the occupied and the virtual orbitals separately to diagonalise the Fock
// blocks (fock and eri rewritten in place)
void semicanonicalize(int n, int nocc, double* fock, double* eri);
}
