/*
 * ccsd_b200.h -- C ABI of the B200 engine for the CCSD amplitude iteration.
 *
 * The engine replaces, for one GPU, the tensor leaf and the irrep-block loop
 * under the reference's indexed-tensor interface
 *   (src/tensor/indexable_tensor.hpp:133-155: mult/sum/scale/dot;
 *    src/tensor/spinorbital_tensor.cxx:455-1109: spin-orbital semantics;
 *    src/tensor/symblocked_tensor.cxx:863-1395: irrep-block loop;
 *    src/tensor/ctf_tensor.cxx:402-514: leaf norm/mult/sum/scale/dot/weight)
 * plus the CCSD iteration driver around it
 *   (src/cc/ccsd.cxx:29-193, src/util/iterative.hpp:126-188,
 *    src/convergence/diis.hpp:70-227, src/operator/denominator.hpp:14-95).
 *
 * Conventions
 *  - Every entry point returns an int status (CCSD_OK = 0); no exception ever
 *    crosses the ABI.  ccsd_last_error() gives a message for the last failure
 *    on a context.
 *  - Spin-orbital tensors follow the reference's SpinorbitalTensor layout:
 *    index positions are ordered [upper vrt, upper occ, lower vrt, lower occ]
 *    (spaces {vrt, occ}, src/operator/2eoperator.cxx:13-21); a spin case is
 *    the number of alpha indices in each of those four groups, alpha indices
 *    first inside a group (src/tensor/spinorbital_tensor.cxx:387-432).
 *  - Within a spin case, blocks are irrep tuples whose XOR is 0 (Abelian
 *    groups C1, C2, C2v/D2 type, D2h: 1, 2, 4 or 8 irreps).
 *  - Dense block storage puts the FIRST index fastest, as the reference's key
 *    convention does (src/tensor/ctf_tensor.hpp:221-226), so a key is the
 *    linear offset inside its block.  Antisymmetric same-spin pairs are stored
 *    unpacked (both orders), except in tensors created CCSD_TENSOR_PACKED,
 *    which store each same-spin pair of a group once (first index < second).
 *  - All calls on a context are ordered on its CUDA stream.  A context is not
 *    thread-safe; several contexts may share a device.
 */
#ifndef CCSD_B200_H
#define CCSD_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    CCSD_OK              = 0,
    CCSD_ERR_ARG         = 1,   /* bad argument / unknown handle / bad index string */
    CCSD_ERR_CUDA        = 2,   /* a CUDA runtime call failed */
    CCSD_ERR_OOM         = 3,   /* device allocation failed or admission refused */
    CCSD_ERR_PLAN        = 4,   /* contraction pattern not supported by the planner */
    CCSD_DIVERGED        = 5,   /* NaN/Inf or runaway residual detected */
    CCSD_NOT_CONVERGED   = 6,   /* max_iter reached without conv < conv_tol */
    CCSD_ERR_SINGULAR    = 7,   /* DIIS system singular after the eps retry (diis.hpp:187) */
    CCSD_ERR_TIMEOUT     = 8,   /* a bounded device wait gave up */
    CCSD_ERR_UNSUPPORTED = 9
};

typedef struct ccsd_ctx_s* ccsd_ctx;
typedef int32_t ccsd_tensor;          /* tensor handle, > 0 */
typedef struct ccsd_solver_s* ccsd_solver;

/* precision of the contraction layer */
enum {
    CCSD_PREC_FP64     = 0,   /* native FP64 GEMMs (plain path) */
    CCSD_PREC_SPLIT    = 1,   /* split BF16 slices on tcgen05, FP32 accumulate, summed in FP64 */
    CCSD_PREC_SPLIT_I8 = 2    /* split INT8 slices on tcgen05 (twice the BF16 rate), exact INT32
                                 accumulate per slice level, summed in FP64 */
};

/* tensor creation flags */
enum {
    CCSD_TENSOR_PACKED = 1,  /* store same-spin antisymmetric pairs once (i<j) */
    /* a plain irrep-blocked tensor over spatial orbitals (the reference's
     * SymmetryBlockedTensor with NS symmetry, src/tensor/symblocked_tensor.cxx): no
     * spin cases, no antisymmetry; contractions among plain tensors are plain
     * einsums.  Positions still follow [upper vrt, upper occ, lower vrt, lower occ],
     * so an index string names the letters in that order; upper and lower counts must
     * be equal. */
    CCSD_TENSOR_PLAIN = 2
};

/* ---- context ------------------------------------------------------------ */
/* stream: a cudaStream_t, or NULL to let the context create its own.  device < 0 makes a
 * planning-only context (no GPU needed): tensors are created and contractions planned and
 * accounted (ccsd_ctx_device_bytes, ccsd_ctx_plan_flops), nothing is launched, and calls
 * that read or write tensor data fail with CCSD_ERR_UNSUPPORTED. */
int ccsd_ctx_create(int device, void* stream, ccsd_ctx* out);
/* algorithmic flops of the last ccsd_contract statement, as the planner counts them
 * (block products 2*M*N*K, packed pairs counted once) */
int ccsd_ctx_plan_flops(ccsd_ctx ctx, double* flops);
/* Diagnostic: write the plan of the last ccsd_contract / ccsd_sum statement on this context
 * (its block GEMMs with their offset tables, permuted sums, block scalings, in execution
 * order) and the block layout of the tensors it touches to a text file, so that a host-side
 * checker can replay the planner's expansion of a statement.  Record format: the header of
 * aquarius_b200/csrc/plan_export.cpp.  Works on planning-only contexts. */
int ccsd_ctx_plan_export(ccsd_ctx ctx, const char* path);
int ccsd_ctx_destroy(ccsd_ctx ctx);
const char* ccsd_last_error(ccsd_ctx ctx);
int ccsd_ctx_synchronize(ccsd_ctx ctx);
/* bytes currently held on the device by this context */
int ccsd_ctx_device_bytes(ccsd_ctx ctx, int64_t* bytes);
/* number of engine kernels launched on this context since creation */
int ccsd_ctx_launch_count(ccsd_ctx ctx, int64_t* count);
/* precision used by subsequent ccsd_contract calls (CCSD_PREC_*); slices=0: default */
int ccsd_ctx_set_precision(ccsd_ctx ctx, int precision, int slices);
/* Which contractions the split precision sends to the tensor-core kernel: AUTO keeps
 * small, skinny or few-tile products on the FP64 kernel; ALL routes every product
 * (coverage of small cases).  The environment variable CCSD_SPLIT_ALL=1 sets ALL at
 * context creation.  ccsd_ctx_split_launches gives the split GEMMs issued so far.
 * No counterpart in the reference (its contractions have one precision). */
enum { CCSD_SPLIT_ROUTE_AUTO = 0, CCSD_SPLIT_ROUTE_ALL = 1 };
int ccsd_ctx_set_split_routing(ccsd_ctx ctx, int mode);
int ccsd_ctx_split_launches(ccsd_ctx ctx, int64_t* launches);
/* Per-statement timing of contraction kernels with CUDA events on the context stream
 * (the role of the reference's named timers, src/time/time.hpp:103-147).  The report is
 * a JSON object {statement: {"launches": n, "ms": t, "flops": f}}; it synchronises the
 * stream and clears the totals.  *needed receives the buffer size required. */
int ccsd_ctx_set_profiling(ccsd_ctx ctx, int on);
int ccsd_ctx_profile_report(ccsd_ctx ctx, char* buf, int64_t buflen, int64_t* needed);

/* Orbital spaces (Space of src/operator/space.hpp): per-irrep counts of
 * alpha/beta virtual and occupied orbitals.  nirrep in {1,2,4,8}.  vrt_beta and
 * occ_beta may be NULL: closed shell, the alpha counts for both spins. */
int ccsd_ctx_set_spaces(ccsd_ctx ctx, int nirrep,
                        const int* vrt_alpha, const int* vrt_beta,
                        const int* occ_alpha, const int* occ_beta);

/* ---- tensors ------------------------------------------------------------ */
/* nout[2], nin[2]: number of upper / lower indices in {vrt, occ}
 * (SpinorbitalTensor ctor, src/tensor/spinorbital_tensor.cxx:166-272) */
int ccsd_tensor_create(ccsd_ctx ctx, const char* name, const int nout[2], const int nin[2],
                       int flags, ccsd_tensor* out);
int ccsd_tensor_destroy(ccsd_ctx ctx, ccsd_tensor t);
int ccsd_tensor_ndim(ccsd_ctx ctx, ccsd_tensor t, int* ndim);
/* number of spin cases; case k has alpha counts alpha[4*k .. 4*k+3] */
int ccsd_tensor_spin_cases(ccsd_ctx ctx, ccsd_tensor t, int* ncases, int* alpha /* 4*ncases or NULL */);
/* element count of one block (spin case + irreps[ndim]) -- 0 if the block is not stored */
int ccsd_tensor_block_size(ccsd_ctx ctx, ccsd_tensor t, const int alpha[4], const int* irreps, int64_t* n);
/* whole-block dense host<->device copies (first index fastest) */
int ccsd_tensor_write_block(ccsd_ctx ctx, ccsd_tensor t, const int alpha[4], const int* irreps,
                            const double* host);
int ccsd_tensor_read_block(ccsd_ctx ctx, ccsd_tensor t, const int alpha[4], const int* irreps,
                           double* host);
/* key/value access inside one block (tCTF_Tensor::write/read, ctf_tensor.hpp:139-247):
 * value <- beta*value + alpha*vals[k] */
int ccsd_tensor_write(ccsd_ctx ctx, ccsd_tensor t, const int alpha_spin[4], const int* irreps,
                      int64_t n, const int64_t* keys, const double* vals, double alpha, double beta);
int ccsd_tensor_read(ccsd_ctx ctx, ccsd_tensor t, const int alpha_spin[4], const int* irreps,
                     int64_t n, const int64_t* keys, double* vals);
/* set every stored element to val */
int ccsd_tensor_fill(ccsd_ctx ctx, ccsd_tensor t, double val);

/* ---- indexed-tensor operations (IndexableTensorBase, indexable_tensor.hpp:133-155) ---- */
/* C[idxC] = beta*C[idxC] + alpha * A[idxA] * B[idxB], with the reference's implicit
 * antisymmetrisation of external lines split between A and B
 * (SpinorbitalTensor::mult, spinorbital_tensor.cxx:455-790).  beta is applied
 * once to every block of C that receives a contribution. */
int ccsd_contract(ccsd_ctx ctx, double alpha, ccsd_tensor A, const char* idxA,
                  ccsd_tensor B, const char* idxB, double beta, ccsd_tensor C, const char* idxC);
/* B[idxB] = beta*B[idxB] + alpha*A[idxA]  (SpinorbitalTensor::sum, spinorbital_tensor.cxx:793-1018) */
int ccsd_sum(ccsd_ctx ctx, double alpha, ccsd_tensor A, const char* idxA,
             double beta, ccsd_tensor B, const char* idxB);
/* A *= alpha  (SpinorbitalTensor::scale) */
int ccsd_scale(ccsd_ctx ctx, ccsd_tensor A, double alpha);
/* full spin-orbital contraction to a scalar (SpinorbitalTensor::dot, :1063-1074) */
int ccsd_dot(ccsd_ctx ctx, ccsd_tensor A, const char* idxA, ccsd_tensor B, const char* idxB, double* out);
/* p = 0 (max-abs), 1 or 2 (SpinorbitalTensor::norm, :1077-1109) */
int ccsd_norm(ccsd_ctx ctx, ccsd_tensor A, int p, double* out);
/* Jacobi weight x /= (sum of index denominators + shift), 0 if |den+shift| < 1e-4
 * (CTFTensor::weight, ctf_tensor.cxx:480-514).  Denominators per spin and irrep,
 * concatenated over irreps: dvrt_a/dvrt_b = -f_aa, docc_a/docc_b = +f_ii
 * (Denominator, denominator.hpp:50-73). */
int ccsd_weight(ccsd_ctx ctx, ccsd_tensor A, const double* dvrt_a, const double* dvrt_b,
                const double* docc_a, const double* docc_b, double shift);

/* ---- CCSD solver (CCSD<U>::run / iterate, Iterative<U>::run, DIIS) -------- */
typedef struct {
    double conv_tol;      /* default 1e-9  (ccsd.cxx:269-270) */
    int    max_iter;      /* default 50    (ccsd.cxx:271-272) */
    int    diis_order;    /* default 5     (ccsd.cxx:281-282) */
    int    diis_start;    /* default 1     (ccsd.cxx:279-280) */
    double diis_damping;  /* default 0.0   (ccsd.cxx:277-278) */
    int    precision;     /* CCSD_PREC_FP64, CCSD_PREC_SPLIT or CCSD_PREC_SPLIT_I8 */
    int    slices;        /* slices per operand: 3 or 4 for BF16, 3, 4 or 5 for INT8
                             (0 = the precision's default) */
    int    use_graph;     /* capture one iteration as a CUDA graph and replay it */
    double refine_tol;    /* split precision only: once conv < refine_tol, 3-slice
                             contractions move to 4 slices; if the residual then stalls,
                             INT8 moves on to 5 slices and then to native FP64 (BF16 from
                             4 slices to FP64) (0 = never).  10 to 1000 x conv_tol, above
                             the 3-slice floor (near 1e-9 for BF16, 4e-7 for INT8 at
                             o=32 v=256); DIIS restarts at every switch */
    double autotune_de;   /* split precision only, > 0: slice count per contraction.  On
                             the first iteration run at 4 or more slices, every statement
                             with split contractions is evaluated once with one slice
                             fewer, from the same amplitudes, and the change of the next
                             energy is measured; statements whose changes add up to at
                             most autotune_de (in Eh, smallest first) keep one slice fewer
                             from then on (0 = every contraction at the solver's count) */
} ccsd_options;

void ccsd_options_default(ccsd_options* opts);

/* The slice autotuner's rule, host only (no counterpart in the reference): given the
 * measured energy changes dE[0..n) of dropping one slice in each of n statements, set
 * drop[i] = 1 for the statements that take one slice fewer: smallest |dE| first, while
 * the sum of the chosen |dE| stays <= budget (ties keep statement order). */
int ccsd_slice_choice(int n, const double* dE, double budget, int* drop);
/* Per statement of the solver's iteration with split contractions: its label, the slices
 * it runs with and the energy change measured by the autotuner (0 if it did not run),
 * as text lines "slices<TAB>dE<TAB>label\n" into buf (len bytes, NUL-terminated; the
 * needed size is returned in *needed). */
int ccsd_solver_slice_report(ccsd_solver s, char* buf, int64_t len, int64_t* needed);

/* The 13 blocks of H in the order of TwoElectronOperator
 * (2eoperator.cxx:13-21, 1eoperator.hpp:39-44):
 *   fAI "ai", fME "ia", fAE "ab", fMI "ij",
 *   VMNIJ "ijkl", VAMIJ "aijk", VMNEJ "ijak", VABIJ "abij", VMNEF "ijab",
 *   VAMEI "aibj", VAMEF "aibc", VABEJ "abci", VABEF "abcd". */
typedef struct {
    ccsd_tensor fAI, fME, fAE, fMI;
    ccsd_tensor VMNIJ, VAMIJ, VMNEJ, VABIJ, VMNEF, VAMEI, VAMEF, VABEJ, VABEF;
} ccsd_hamiltonian;

/* Build the 13 H blocks on the device from a three-index factor
 * (pq|rs) = sum_P B[P,p,q] B[P,r,s] (closed shell, spatial orbitals shared by
 * both spins) and a diagonal Fock matrix eps[n].  Orbitals are ordered occupied
 * first, irrep-major inside occ and vrt, matching ccsd_ctx_set_spaces.
 * B is a host array [naux][n][n]; aux_per_irrep (may be NULL) gives the irrep
 * split of P so that each block only sums over the P of matching irrep.
 * pack_vvvv != 0 stores VABEF with packed same-spin pairs (halves its memory). */
int ccsd_hamiltonian_from_factor(ccsd_ctx ctx, int naux, const double* B, const double* eps,
                                 const int* aux_per_irrep, int pack_vvvv, ccsd_hamiltonian* H);
int ccsd_hamiltonian_destroy(ccsd_ctx ctx, ccsd_hamiltonian* H);

/* The 13 H blocks, zero-filled, for the caller to write (ccsd_tensor_write_block /
 * ccsd_tensor_write): the TwoElectronOperator constructor (src/operator/2eoperator.cxx:10-21)
 * that an integral transformation (src/operator/aomoints.cxx) then fills.  Any spaces,
 * open shell included.  <ij||ak>, <ab||ij> and <ab||ci> are views of <ai||jk>, <ij||ab>
 * and <ai||bc> (Hermiticity): write those three and the views follow. */
int ccsd_hamiltonian_create(ccsd_ctx ctx, int pack_vvvv, ccsd_hamiltonian* H);

/* Closed-shell H from dense spatial integrals (the assembly of src/operator/fcidump.cxx:472-514):
 * fock[n*n] (row = upper index), eri[n^4] = (pq|rs) in chemists' notation, last index
 * fastest; orbitals occupied first, irrep-major inside occ and vrt as in
 * ccsd_ctx_set_spaces (alpha = beta, n = occ + vrt). */
int ccsd_hamiltonian_from_integrals(ccsd_ctx ctx, int n, const double* fock, const double* eri, int pack_vvvv,
                                    ccsd_hamiltonian* H);

/* FCIDUMP input (src/operator/fcidump.cxx:35-516, task "fcidump"; options
 * "1eints full" and "semicanonical"). */
enum {
    CCSD_FCIDUMP_FULL_FOCK = 1,      /* one-electron records are the full matrix (no mirroring) */
    CCSD_FCIDUMP_SEMICANONICAL = 2   /* diagonalise the occupied and virtual Fock blocks */
};
/* Parse a file on the host.  h (n*n) and eri (n^4, dense, all eight images filled) may
 * be NULL: then only NORB / NELEC are read.  No device needed. */
int ccsd_fcidump_read(const char* path, int flags, int* norb, int* nelec, double* ecore, double* h, double* eri);
/* Read a file, set the context's spaces (C1, NELEC/2 occupied, closed shell), build the
 * Fock matrix and H on the device; escf (may be NULL) receives E_core + sum_i (h_ii + f_ii). */
/* Closed shell from AO quantities (the integral transformation of aomoints.cxx:1017-1450 /
 * rhfaomoints.cxx:37-180): hcore[nao*nao] and the AO integrals eri_ao[nao^4] = (mu nu|la si)
 * (last index fastest), MO coefficients C[nao*nmo] (row-major, column p = MO p, occupied
 * first).  The MO integrals are formed on the device (four quarter transformations on the
 * FP64 GEMM kernels), the MO Fock matrix from them, then H as ccsd_hamiltonian_from_integrals
 * does.  Sets C1 spaces (nocc occupied, nmo - nocc virtual) on a context without tensors.
 * *e_elec (optional) receives sum_i (h_ii + f_ii), the SCF electronic energy of C.  The AO
 * array is held on the device (nao^4 + nmo nao^3 doubles); nao^3 must stay below 2^23. */
int ccsd_hamiltonian_from_ao(ccsd_ctx ctx, int nao, int nmo, int nocc, const double* hcore, const double* eri_ao,
                             const double* C, int pack_vvvv, ccsd_hamiltonian* H, double* e_elec);
int ccsd_hamiltonian_from_fcidump(ccsd_ctx ctx, const char* path, int flags, int pack_vvvv, ccsd_hamiltonian* H,
                                  double* escf);

/* Solver: allocates T, Z, Tau, the 7 intermediates and the DIIS ring, forms the
 * MP1 guess and the MP2 energy (ccsd.cxx:37-62), and plans one iteration. */
int ccsd_solver_create(ccsd_ctx ctx, const ccsd_hamiltonian* H, const ccsd_options* opts,
                       ccsd_solver* out);

/* ---- closed-shell spin-adapted CCSD (RHFCCSD, src/cc/rhfccsd.cxx) --------------
 * The same iteration driver over plain spatial tensors (CCSD_TENSOR_PLAIN): about
 * half the flops of the spin-orbital form for a closed-shell reference.  The blocks
 * are the non-antisymmetrised <pq|rs> of the reference's RHF integrals; positions
 * follow the tensor layout [upper vrt, upper occ, lower vrt, lower occ], so VAIJB
 * stores <ai|jb> at [a, i, b, j].  fAI, fAB and fIJ are the Fock blocks. */
typedef struct {
    ccsd_tensor fAI, fAB, fIJ, VABCD, VABCI, VABIJ, VAIBJ, VAIJB, VAIJK, VIJKL;
} ccsd_rhf_hamiltonian;
/* from a three-index factor (arguments as ccsd_hamiltonian_from_factor) */
int ccsd_rhf_hamiltonian_from_factor(ccsd_ctx ctx, int naux, const double* B, const double* eps,
                                     const int* aux_per_irrep, ccsd_rhf_hamiltonian* H);
/* from a spatial Fock matrix and dense (pq|rs) (arguments as ccsd_hamiltonian_from_integrals) */
int ccsd_rhf_hamiltonian_from_integrals(ccsd_ctx ctx, int n, const double* fock, const double* eri,
                                        ccsd_rhf_hamiltonian* H);
/* from AO quantities (arguments as ccsd_hamiltonian_from_ao) */
int ccsd_rhf_hamiltonian_from_ao(ccsd_ctx ctx, int nao, int nmo, int nocc, const double* hcore,
                                 const double* eri_ao, const double* C, ccsd_rhf_hamiltonian* H, double* e_elec);
int ccsd_rhf_hamiltonian_destroy(ccsd_ctx ctx, ccsd_rhf_hamiltonian* H);
/* Solver over the RHF blocks: RHFCCSD::run / iterate (rhfccsd.cxx:44-110, 193-327); the
 * solver handle then works with every ccsd_solver_* call (amplitudes are plain tensors) */
int ccsd_rhf_solver_create(ccsd_ctx ctx, const ccsd_rhf_hamiltonian* H, const ccsd_options* opts,
                           ccsd_solver* out);
/* host-only plan of one RHF iteration: flops and peak device bytes (as ccsd_plan_query) */
int ccsd_rhf_plan_query(int nirrep, const int* vrt, const int* occ, const ccsd_options* opts,
                        double* flops_per_iter, int64_t* device_bytes);
int ccsd_solver_destroy(ccsd_solver s);
int ccsd_solver_mp2(ccsd_solver s, double* mp2);
/* one CCSD::iterate; energy and conv (max-abs of the weighted update) come back to the host */
int ccsd_solver_iterate(ccsd_solver s, double* energy, double* conv);
/* one iteration without reading energy/conv back (stream-ordered, no host sync) */
int ccsd_solver_iterate_async(ccsd_solver s);
/* read the energy / convergence of the last iteration (synchronises the stream) */
int ccsd_solver_status(ccsd_solver s, double* energy, double* conv, int* iterations);
/* Iterative::run: iterate until conv < conv_tol or max_iter */
int ccsd_solver_run(ccsd_solver s, double* energy, double* conv, int* iterations);
/* amplitudes T1 / T2 as tensors of the solver (for reading) */
int ccsd_solver_amplitudes(ccsd_solver s, ccsd_tensor* T1, ccsd_tensor* T2);
/* Closed-shell similarity-transformed Hamiltonian intermediates after convergence
 * (RHFCCSD::run "Form Hbar", rhfccsd.cxx:110-186) from the solver's current T1, T2: plain
 * tensors owned by the solver (valid until it is destroyed; recomputed on every call).
 * WAMIE keeps the engine's [a, m, e, i] position order for the reference's (a, m, i, e). */
typedef struct {
    ccsd_tensor FME, FMI, FAE, WMNIJ, WMNEJ, WAMIJ, WAMIE, WAMEI, WABEJ;
} ccsd_rhf_hbar;
int ccsd_rhf_solver_hbar(ccsd_solver s, ccsd_rhf_hbar* out);
/* Spin-orbital similarity-transformed Hamiltonian after convergence: the "Hbar" product of
 * CCSD::run (ccsd.cxx:83-86), STTwoElectronOperator(H, T, isHbar) for T truncated at doubles
 * (st2eoperator.hpp:59-130), from the solver's current T1, T2.  Thirteen blocks of the
 * solver's own (valid until it is destroyed; recomputed on every call, which fails while a
 * Lambda solver reads them).  As in the reference: fAI and VABIJ are zero, fME holds only
 * sum_nf <mn||ef> t_fn (the bare f_me is replaced: zero for an SCF reference), and no block
 * is a view of another.  Needs the solver's <ab||ef> stored unpacked (pack_vvvv = 0):
 * otherwise CCSD_ERR_UNSUPPORTED.  Replaces LambdaCCSD's requirement "ccsd.Hbar". */
int ccsd_solver_hbar(ccsd_solver s, ccsd_hamiltonian* out);

/* Lambda-CCSD (LambdaCCSD<U>::run / iterate, src/cc/lambdaccsd.cxx:27-133) on an Hbar
 * (normally from ccsd_solver_hbar) and the amplitudes of the spin-orbital CCSD solver
 * `ccsd` (T2 is read every iteration by G(im), G(ea); destroying `ccsd` first fails).
 * The returned handle works with ccsd_solver_iterate / _iterate_async / _status / _run /
 * _destroy: the energy is 1/4 <mn||ef> l_mn^ef (lambdaccsd.cxx:129), conv the max-abs of
 * the weighted update, ccsd_solver_amplitudes gives L1 [i, a] and L2 [i, j, a, b] (upper
 * occupied, lower virtual), and ccsd_solver_mp2 the energy of the initial guess L = T.
 * The denominators are the diagonals of Hbar's fAE and fMI (Denominator(Hbar)). */
int ccsd_lambda_solver_create(ccsd_ctx ctx, const ccsd_hamiltonian* hbar, ccsd_solver ccsd,
                              const ccsd_options* opts, ccsd_solver* out);
/* host-only plan of CCSD + Hbar + Lambda in C1 or D2h sizes: flops of forming Hbar, flops
 * of one Lambda iteration and the peak device bytes with all three alive */
int ccsd_lambda_plan_query(int nirrep, const int* vrt, const int* occ, const ccsd_options* opts,
                           double* hbar_flops, double* flops_per_iter, int64_t* device_bytes);
/* Diagnostic: plan a solver on the host for C1 or D2h sizes (unpacked <ab||ef>) and write
 * one of its recorded plans in the format of ccsd_ctx_plan_export, so that a host-side
 * checker can replay the solver's statement list.  vrt_beta / occ_beta may be NULL (closed
 * shell; must be NULL for CCSD_METHOD_RHF).  method: CCSD_METHOD_*; which:
 * CCSD_PLAN_ITERATION (the Tau statements, then one iteration's intermediates and
 * residual), CCSD_PLAN_HBAR (CCSD and RHF only) or CCSD_PLAN_ENERGY. */
enum { CCSD_METHOD_CCSD = 0, CCSD_METHOD_RHF = 1, CCSD_METHOD_LAMBDA = 2 };
enum { CCSD_PLAN_ITERATION = 0, CCSD_PLAN_HBAR = 1, CCSD_PLAN_ENERGY = 2 };
int ccsd_plan_export_solver(int method, int nirrep, const int* vrt, const int* occ, const int* vrt_beta,
                            const int* occ_beta, int which, const char* path);
/* algorithmic FP64 flops of one iteration as planned (packed-pair counts) */
int ccsd_solver_flops(ccsd_solver s, double* flops);
/* contraction mode the next iteration uses (changes when refine_tol is reached):
 * CCSD_PREC_* and, for the split precision, the BF16 slices per operand */
int ccsd_solver_mode(ccsd_solver s, int* precision, int* slices);

/* Planning query, host only (no device is touched): algorithmic FP64 flops of one
 * iteration (reference flop convention: packed same-spin pairs count once) and the
 * device bytes a solve of these spaces needs (H + amplitudes + intermediates + DIIS
 * ring + plan tables; the peak of the factor build included).  Serves admission by
 * HBM footprint.  Closed-shell spaces: alpha = beta counts. */
int ccsd_plan_query(int nirrep, const int* vrt_per_irrep, const int* occ_per_irrep, const ccsd_options* opts,
                    int pack_vvvv, double* flops_per_iter, int64_t* device_bytes);

/* ---- DIIS over caller tensors ------------------------------------------------
 * DIIS<T> of src/convergence/diis.hpp:36-228: its constructor (order, start, damping) and
 * extrapolate(x, dx) (:70-227), which CCSD<U>::iterate calls at src/cc/ccsd.cxx:192; for
 * a caller that keeps its own iteration (the solvers run the same DIIS internally).
 * A vector is the concatenation of n tensor pieces (e.g. {T1, T2}): x[k] and dx[k] have
 * the same shape, and every call passes pieces of the first call's shapes.  The inner
 * product is sum_k w_k <a_k, b_k> over full spin-orbital ranges, with w_k = weights[k],
 * or, for weights NULL, 1 / (upper! lower!) of piece k: 1 for T1 and 1/4 for T2, as
 * ExcitationOperator::dot (src/operator/excitationoperator.hpp:77-87); plain tensors 1.
 * Each call stores copies of x and dx in a device ring of `order` pairs, adds the new
 * error-matrix row, and once two pairs are stored and the start counter allows it solves
 * the bordered system (Lagrange row -1, an eps-shifted retry when singular) and overwrites
 * x and dx with sum c_i x_i and sum c_i dx_i; otherwise x and dx keep their values.
 * damping > 0 applies the reference's damping of the stored newest x while the start
 * counter is above 1.  The call synchronises the context's stream and returns
 * CCSD_ERR_SINGULAR if the system stays singular.  Packed tensors are refused.  Destroy
 * the DIIS object before its context. */
typedef struct ccsd_diis_s* ccsd_diis;
int ccsd_diis_create(ccsd_ctx ctx, int order, int start, double damping, ccsd_diis* out);
int ccsd_diis_extrapolate(ccsd_diis d, int n, const ccsd_tensor* x, const ccsd_tensor* dx, const double* weights);
/* coefficients of the last extrapolation by age (c[0]: the pair just stored), `order`
 * entries; *nvec = stored pairs (c is a unit vector when no extrapolation happened) */
int ccsd_diis_coefficients(ccsd_diis d, int* nvec, double* c);
int ccsd_diis_destroy(ccsd_diis d);

/* ---- allocation-free variant -------------------------------------------------
 * No counterpart in the reference.  out[j] = <x, ys[j]> for j < ny, the batched dot of
 * the DIIS error-matrix row, for callers that must not have the library allocate device
 * memory (an application that owns all device memory through its own arena or pool and
 * forbids libraries to allocate behind its back).  x, every ys[j] (n doubles each) and out
 * (ny doubles) are caller-owned device buffers on the current device; ys itself is a
 * HOST array of ny device pointers; work is ordered on `stream` (a cudaStream_t, NULL
 * for the default stream) and the call does not synchronise.  The partial sums live in
 * a fixed 32 KiB device array inside the library: ny is limited to 1..16 (else
 * CCSD_ERR_ARG, message in ccsd_last_error(NULL)); calls whose kernels overlap on the
 * GPU share that array and race, so serialise them; the first call on a device looks
 * the array up with cudaGetSymbolAddress and should precede any stream capture; that
 * address does not survive cudaDeviceReset.  A CUDA error pending from earlier work is
 * reported (CCSD_ERR_CUDA) and left in place, and nothing is launched. */
int ccsd_dot_batch_noalloc(void* stream, const double* x, const double* const* ys, int ny, int64_t n,
                           double* out);

/* ---- serving: continuous batching of solves on one device ------------------
 * No counterpart in the reference (it runs one solve per job).  Requests of any size
 * are queued on submission; an admission thread takes them in arrival order as soon as
 * their planned device bytes (ccsd_plan_query) fit in the memory budget next to the
 * active solves and a slot is free, and starts a worker thread for each.  The worker
 * builds H on a context and stream of its own and runs the iterations back to back,
 * sleeping on each iteration's completion event, until the residual is below conv_tol
 * or max_iter is reached; then it frees the solve's memory for the next admission.  The
 * iterations of all active solves overlap on the device through their streams.  Every
 * solve's kernels and reductions are those of a lone solve, so its result does not
 * depend on the mix. */
typedef struct ccsd_server_s* ccsd_server;
typedef struct {
    int device;
    int64_t memory_budget;   /* bytes the active solves may hold; 0: 90% of the free memory */
    int max_active;          /* concurrent solves; 0: 16 */
    int pack_vvvv;
    ccsd_options solve;      /* per-solve options (precision, conv_tol, max_iter, DIIS, ...) */
} ccsd_server_options;
typedef struct {
    int64_t id;
    int status;              /* CCSD_OK, CCSD_NOT_CONVERGED or the error of the solve */
    int iterations;
    double energy, mp2, conv;
    double t_submit, t_admit, t_done;   /* seconds since the server started */
    int64_t device_bytes;    /* planned bytes the solve was admitted with */
    double flops_per_iter;
    int64_t peak_bytes;      /* device bytes the solve's context held at its peak */
    double t_built;          /* when its H and solver were ready (seconds since the server started) */
    char message[160];       /* the error message of a failed solve ("" otherwise) */
} ccsd_server_result;
void ccsd_server_options_default(ccsd_server_options* o);
int ccsd_server_create(const ccsd_server_options* o, ccsd_server* out);
/* a synthetic request (the seeded generator below, o and v split over nirrep irreps) */
int ccsd_server_submit_synthetic(ccsd_server s, int nirrep, int o, int v, uint64_t seed, int64_t* id);
/* a request from a three-index factor (copied; arguments as ccsd_hamiltonian_from_factor) */
int ccsd_server_submit_factor(ccsd_server s, int nirrep, const int* vrt, const int* occ, int naux, const double* B,
                              const double* eps, const int* aux_per_irrep, int64_t* id);
/* move up to max finished results into out (non-blocking); *n receives their count */
int ccsd_server_poll(ccsd_server s, int max, ccsd_server_result* out, int* n);
/* block until every submitted request has finished or timeout_s passed (CCSD_ERR_TIMEOUT) */
int ccsd_server_wait(ccsd_server s, double timeout_s);
/* requests queued, solves active, peak bytes admitted at once, peak solves active at once */
int ccsd_server_stats(ccsd_server s, int* queued, int* active, int64_t* peak_bytes, int* peak_active);
int ccsd_server_destroy(ccsd_server s);

/* ---- synthetic inputs (seeded; identical on every host) -------------------- */
/* irrep sizes: Dirichlet(1.5) split of o, v and naux = 3(o+v) (aux may be NULL) */
int ccsd_synth_irreps(uint64_t seed, int nirrep, int o, int v,
                      int* occ_per_irrep, int* vrt_per_irrep, int* aux_per_irrep);
/* eps[n] (n = o+v) and B[naux][n][n] (either may be NULL) */
int ccsd_synth_problem(uint64_t seed, int nirrep,
                       const int* occ_per_irrep, const int* vrt_per_irrep, const int* aux_per_irrep,
                       double* eps, double* B);

#ifdef __cplusplus
}
#endif
#endif
