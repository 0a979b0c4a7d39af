// CCSD solver state (see solver.cpp).
#pragma once
#include <vector>
#include <utility>

#include "engine.hpp"

namespace ccsd {

void options_default(ccsd_options* o);
// the slice autotuner's rule: 1 for the statements that take one slice fewer
std::vector<int> slice_choice(const std::vector<double>& dE, double budget);

struct DiisSegment {
    int64_t off, len;
    double w;
};

class Solver {
public:
    Context& ctx;
    ccsd_hamiltonian H{};              // spin-orbital blocks (ccsd.cxx)
    ccsd_rhf_hamiltonian HR{};         // closed-shell spatial blocks (rhfccsd.cxx)
    bool rhf = false;
    ccsd_options opts;
    int T1 = 0, T2 = 0, Z1 = 0, Z2 = 0, Tau = 0;
    int FME = 0, FMI = 0, FAE = 0, WMNIJ = 0, WMNEJ = 0, WAMIJ = 0, WAMEI = 0;
    // RHF only: spin-adapted combinations, the extra ring intermediate, and the copies
    // that the in-place symmetrisations WMNIJ += WMNIJ(nmji), Z2 += Z2(baji) read
    int T2SA = 0, TauSA = 0, VABIJSA = 0, VAIJBSA = 0, WAMIE = 0, WMNIJc = 0, Z2c = 0;
    int WABEJ = 0;                     // RHF Hbar only (created on the first hbar())
    // Spin-orbital Hbar (STTwoElectronOperator with isHbar, st2eoperator.hpp:59-130): 13
    // blocks of the solver's own, created on the first hbar_so()
    ccsd_hamiltonian HB{};
    bool hbar_formed = false;
    // Lambda-CCSD (lambdaccsd.cxx): H holds the Hbar blocks, T1/T2/Z1/Z2 are L(1)[ia],
    // L(2)[ijab] and their updates, `source` is the CCSD solver whose T2 G(im)/G(ea) read
    bool lambda = false;
    int GIM = 0, GEA = 0;
    Solver* source = nullptr;
    int lambda_users = 0;              // Lambda solvers reading this solver's T and Hbar
    Plan hbar_plan;
    double* den[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [space][spin]
    Plan iter_plan, tau_plan, energy_plan;
    double* d_red = nullptr;    // [0] energy, [1] conv
    double* h_red = nullptr;
    int* h_state = nullptr;
    // DIIS
    std::vector<double*> xs, dxs;
    const double** d_xs = nullptr;
    const double** d_dxs = nullptr;
    double *d_e = nullptr, *d_c = nullptr, *d_dots = nullptr;
    int* d_state = nullptr;
    int64_t vec_len = 0;
    std::vector<DiisSegment> segs;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool captured_once = false;
    bool refined = false;           // moved to a more accurate contraction mode (refine_tol reached)
    // this solver's contraction mode (precision, slices): the context's routing fields are
    // shared by every solver on it, so each entry point that launches contractions first
    // puts the solver's own mode in place (use_mode) and a refinement switch updates it
    int mode_precision = CCSD_PREC_FP64, mode_slices = 0;
    // slice autotuner (opts.autotune_de): per statement label, measured energy change and
    // the slice delta chosen
    struct TuneEntry {
        std::string label;
        double dE;
        int delta;
    };
    bool tuned = false;
    std::vector<TuneEntry> tune_report;
    void autotune_slices();
    void use_mode() {
        ctx.precision = mode_precision;
        ctx.slices = mode_slices;
    }
    std::vector<double> conv_hist;  // residuals since the last mode switch (stall detection)
    std::vector<kern::TauArgs> tau_blocks;
    // one-launch Tau and Jacobi update over all blocks: device descriptors and chunk starts
    kern::TauArgs* d_tau = nullptr;
    int64_t* d_tau_cs = nullptr;
    int64_t tau_chunks = 0;
    kern::UpdateDesc* d_upd = nullptr;
    int64_t* d_upd_cs = nullptr;
    int64_t upd_chunks = 0;
    int n_upd = 0;

    int iterations = 0;
    double energy = 0, conv = 0, mp2 = 0;
    double flops_per_iter = 0;
    std::vector<std::pair<void*, size_t>> owned;
    bool constants_registered = false;   // setup() marked constants() as constant tensors

    Solver(Context& c, const ccsd_hamiltonian& h, const ccsd_options& o);
    Solver(Context& c, const ccsd_rhf_hamiltonian& h, const ccsd_options& o);
    // Lambda-CCSD on an Hbar and the amplitudes of a spin-orbital CCSD solver
    Solver(Context& c, Solver& ccsd, const ccsd_hamiltonian& hbar, const ccsd_options& o);
    ~Solver();
    void iterate(double* e, double* c);
    void iterate_async();
    void read_status();
    // read_status in two halves: queue the copies of energy / residual / DIIS state to
    // the host on the context stream, and, once the stream has passed them, check them
    void post_status();
    void check_status();
    int run(double* e, double* c, int* it);
    // closed-shell Hbar intermediates from the current amplitudes (rhfccsd.cxx:110-186)
    void hbar_rhf();
    // spin-orbital Hbar from the current amplitudes into HB
    void hbar_so();

private:
    void* alloc(size_t bytes);
    void build_denominators();
    void build_diis();
    kern::WeightArgs weight_args(const Tensor& T, int cs, const Block& b) const;
    void weight_tensor(int h);
    void record_tau(Plan& p);
    void build_tau_blocks();
    void launch_tau();
    void build_update();
    void record_energy(Plan& p);
    void record_iteration();
    void record_iteration_rhf();
    void record_iteration_lambda();
    void record_hbar_so();
    void setup();
    void setup_or_teardown();
    void teardown();
    std::vector<int> constants() const;
    std::vector<int> owned_tensors() const;
    void launch_iteration();
    void diis_step();
};

}  // namespace ccsd
