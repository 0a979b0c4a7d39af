// Host-side engine: device tensors, the statement planner and the step executor.
//
// The planner reproduces, once per statement, what the reference recomputes on
// every call: the spin-case expansion of SpinorbitalTensor::mult/sum
// (src/tensor/spinorbital_tensor.cxx:455-1018) and the irrep-block walk of
// SymmetryBlockedTensor::mult/sum (src/tensor/symblocked_tensor.cxx:863-1223).
// Its output is a list of steps (block GEMMs with gather/scatter tables,
// strided block sums, scalings) that the executor replays on a CUDA stream.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <functional>
#include <map>
#include <memory>
#include <memory>
#include <stdexcept>

#include <cuda_runtime.h>

#include "ccsd_b200.h"
#include "kernels.hpp"

namespace ccsd {

// device bytes the sliced constant operands may occupy (CCSD_SPLIT_CACHE_GB, default 50)
int64_t split_cache_budget();

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CCSD_CUDA(call)                                                                  \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            throw ::ccsd::Error(CCSD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

enum { VRT = 0, OCC = 1 };
enum { ALPHA = 0, BETA = 1 };

// group g of a spin-orbital tensor: 0 upper vrt, 1 upper occ, 2 lower vrt, 3 lower occ
inline int group_space(int g) { return g % 2 == 0 ? VRT : OCC; }

struct Spaces {
    int nirrep = 1;
    int n[2][2][8] = {};          // [space][spin][irrep]
    int off[2][2][8] = {};        // offset of irrep inside the spin-space range
    int total(int space, int spin) const {
        int s = 0;
        for (int h = 0; h < nirrep; h++) s += n[space][spin][h];
        return s;
    }
};

struct Block {
    std::vector<int> irrep;       // per position
    std::vector<int> len;         // per position
    std::vector<int64_t> stride;  // per position (unpacked dims); packed pairs handled via pair_* fields
    int64_t offset = 0;           // element offset in the tensor storage
    int64_t size = 0;
    // packed pairs (adjacent positions p, p+1 of one group, same spin) stored once in
    // canonical order: kind 1 = triangle x<y (equal irreps), kind 2 = rectangle (irrep p < irrep q)
    struct Pair {
        int p = -1, q = -1;
        int kind = 0;
        int64_t stride = 0;
    };
    std::vector<Pair> pairs;
    int pair_of(int pos) const {
        for (size_t i = 0; i < pairs.size(); i++)
            if (pairs[i].p == pos || pairs[i].q == pos) return (int)i;
        return -1;
    }
};

struct SpinCase {
    int alpha[4] = {0, 0, 0, 0};  // alpha count per group
    std::vector<int> spin;        // per position
    std::vector<Block> blocks;
    std::map<std::vector<int>, int> block_of;   // irreps -> block index (only stored blocks)
};

struct Tensor {
    std::string name;
    int nout[2] = {0, 0}, nin[2] = {0, 0};
    int ndim = 0;
    int flags = 0;
    std::vector<int> group;       // per position
    std::vector<SpinCase> cases;
    double* data = nullptr;       // device
    int64_t total = 0;
    int view_of = 0;              // > 0: blocks alias the storage of that tensor (no own data)

    int find_case(const int alpha[4]) const {
        for (size_t c = 0; c < cases.size(); c++) {
            bool ok = true;
            for (int g = 0; g < 4; g++) ok &= cases[c].alpha[g] == alpha[g];
            if (ok) return (int)c;
        }
        return -1;
    }
    bool packed() const { return flags & CCSD_TENSOR_PACKED; }
    bool plain() const { return flags & CCSD_TENSOR_PLAIN; }
};

// ---------------------------------------------------------------------------
// planned steps
// ---------------------------------------------------------------------------

// One block contraction lowered to GEMM form:
//   for every destination variant v (sign s_v):
//     C[offCm_v[m] + offCn_v[n]] += s_v * alpha * sum_k A[offAm[m]+offAk[k]] * B[offBk[k]+offBn[n]]
struct GemmStep {
    int tA = 0, tB = 0, tC = 0;        // tensor handles (for slicing caches / constness)
    int M = 0, N = 0, K = 0;
    double alpha = 0;
    int nvm = 1, nvn = 1;              // destination variants along m and n
    double vsign[4] = {1, 1, 1, 1};    // sign of variant (im * nvn + in)
    // host copies (for planning / flop counts) and device tables
    std::vector<int64_t> hAm, hAk, hBk, hBn, hCm[2], hCn[2];
    int64_t *dAm = nullptr, *dAk = nullptr, *dBk = nullptr, *dBn = nullptr;
    int64_t *dCm[2] = {nullptr, nullptr}, *dCn[2] = {nullptr, nullptr};
    bool a_mcontig = false, a_kcontig = false, b_kcontig = false, b_ncontig = false;
    // k tables found to be arithmetic progressions at upload (Ak[k] = ak0 + k * ak_step)
    bool ak_affine = false, bk_affine = false;
    int64_t ak0 = 0, ak_step = 0, bk0 = 0, bk_step = 0;
    double flops() const { return 2.0 * M * N * (double)K; }
    std::string label;                 // statement this block contraction came from
    int slice_delta = 0;               // split path: slices relative to the context's count (autotuner)
    bool uploaded = false;             // device tables placed (Context::upload)
    // what the rows, columns and k range of this block product are (operand, spin and irrep
    // of every index, restricted pairs): block products of one statement that share a key
    // along a dimension share those rows / columns / k (merged symmetry-blocked products)
    std::string mkey, nkey, kkey;
    int64_t split_cache_a = -1;        // keys of cached slices of constant operands
    int64_t split_cache_b = -1;
    bool cache_a = false, cache_b = false;   // operand slices kept across calls (set at reserve)
};

// C[perm] += alpha * A  over one block (strided, up to 8 dims)
struct SumStep {
    std::string label;
    int tA = 0, tC = 0;
    int ndim = 0;
    int64_t len[8];
    int64_t sA[8], sC[8];
    int64_t offA = 0, offC = 0;
    double alpha = 0;
};

// C_block *= beta (beta == 0: zero-fill)
struct ScaleStep {
    std::string label;
    int tC = 0;
    int64_t off = 0, n = 0;
    double beta = 1;
};

// scalar += alpha * sum A_blk[x] * B_blk[perm x]  (strided)
struct DotStep {
    int tA = 0, tB = 0;
    int ndim = 0;
    int64_t len[8];
    int64_t sA[8], sB[8];
    int64_t offA = 0, offB = 0;
    double alpha = 0;
};

struct Step {
    enum Kind { GEMM, SUM, SCALE, DOT } kind;
    int idx;                           // index into the typed vector of the plan
};

// tensor handle standing for the plan's scratch product buffer
constexpr int kScratch = -1;

// One launch inside a run of consecutive steps of one kind and one statement: a single
// step, or one batched launch over several steps whose outputs are disjoint (GEMMs on the
// grouped tiled-FP64 kernel, permuted sums, block scalings).
struct GemmLaunch {
    enum Kind { GEMM, GEMM_GROUPED, FOLD_GROUPS, SUM, SUM_BATCHED, SCALE, SCALE_BATCHED, DOT_BATCHED, MERGED_SPLIT,
                SHORT_GROUPED, SKINNY_GROUPED, MERGED_SLICE };
    Kind kind = GEMM;
    int gemm = -1;                     // single GEMM: index into Plan::gemms
    int step = -1;                     // single SUM / SCALE: index into Plan::sums / scales
    bool ak = false, bk = false;       // grouped GEMM: operand contiguity
    int mt = 0, nt = 0;                // short products: fragment shape (d_desc: ShortDesc[nprob]);
                                       // grouped skinny: nt n-groups, ak = L contiguous along k
                                       // (d_desc: SkinnyArgs[nprob])
    int nprob = 0, tiles = 0;
    kern::GemmArgs* d_probs = nullptr;
    int* d_tile_start = nullptr;
    double* d_part = nullptr;          // shared-output group: partial products (part_elems doubles)
    int64_t part_elems = 0;
    int ngroups = 0;                   // fold: output blocks (d_desc: FoldDesc[nprob], d_tile_start: group starts)
    void* d_desc = nullptr;            // batched sums / scalings: descriptors
    int64_t* d_chunks = nullptr;       // ... and their first chunks
    size_t desc_bytes = 0;
    int64_t chunks = 0;
    double flops = 0;
    std::shared_ptr<struct MergedProduct> merged;   // MERGED_SPLIT
    void* arena = nullptr;             // batched slicing of merged products: their operands'
    size_t arena_bytes = 0;            // slices, scales and row maxima (aux: the row maxima)
    void* aux = nullptr;
    size_t aux_bytes = 0;
};
// The block products of one irrep class of a symmetry-blocked statement as one dense split
// GEMM: rectangles of A (rows x k), of B (columns x k) and of C (rows x columns) placed in
// the merged operands; the scatter of C runs in levels so that no two rectangles of one
// launch write the same block.
struct MergedProduct {
    int M = 0, N = 0, K = 0;
    int first_gemm = -1;               // a member (slice count)
    int nA = 0, nB = 0;
    int64_t tilesA = 0, tilesB = 0;
    kern::RectDesc* dA = nullptr;
    kern::RectDesc* dB = nullptr;
    int64_t *dA_ts = nullptr, *dB_ts = nullptr;
    struct Level {
        kern::ScatterDesc* d = nullptr;
        int64_t* cs = nullptr;
        int n = 0;
        int64_t chunks = 0;
    };
    std::vector<Level> levels;
    int members = 0;
    // constant operands (the H blocks) keep their sliced rectangles from call to call
    // within the split cache budget; a deeper cached slicing serves fewer slices
    bool cache_a = false, cache_b = false;
    int64_t cache_bytes = 0;           // reserved for both at build
    kern::SlicedOperand sA, sB;
    // the other operands are sliced by one batched launch for all merged products of the
    // statement (MERGED_SLICE, before the first of them) into their own operand buffers
    std::vector<kern::RectDesc> hA, hB;   // host copies of the rectangles
    // each rectangle's host row and k tables (its block product's), to find equal operands
    std::vector<std::pair<const std::vector<int64_t>*, const std::vector<int64_t>*>> srcA, srcB;
    bool self_read = false;            // an operand is the statement's output (no batching)
    bool batched_a = false, batched_b = false;
    kern::SlicedOperand pa, pb;
};
struct GemmRun {
    int first = 0, end = 0;            // steps [first, end)
    std::vector<GemmLaunch> launches;
};
// the grouped schedule of a plan under one routing (precision, split routing, kernels)
struct RunSchedule {
    std::vector<GemmRun> runs;
    std::vector<int> run_at;           // per step: index of the run starting there, or -1
};

struct Plan {
    int64_t scratch_elems = 0;         // doubles of scratch the steps need (products X)
    double* scratch = nullptr;         // allocated at upload
    bool split_reserved = false;       // split-path workspace sized for this plan
    std::vector<std::pair<void*, size_t>> table_pool;   // device buffers holding the steps' tables
    std::vector<Step> steps;
    std::vector<GemmStep> gemms;
    std::vector<SumStep> sums;
    std::vector<ScaleStep> scales;
    std::vector<DotStep> dots;
    std::map<int, RunSchedule> schedules;   // grouped launches per routing key (built on first run)
    double flops() const {
        double f = 0;
        for (auto& g : gemms) f += g.flops();
        return f;
    }
    void append(Plan&& other);
};

class Context;

// Plans C[idxC] = beta C + alpha A[idxA] B[idxB]  (B may be 0 for a sum)
Plan plan_contract(Context& ctx, double alpha, int A, const std::string& idxA, int B, const std::string& idxB,
                   double beta, int C, const std::string& idxC);
Plan plan_sum(Context& ctx, double alpha, int A, const std::string& idxA, double beta, int C,
              const std::string& idxC);
Plan plan_dot(Context& ctx, int A, const std::string& idxA, int B, const std::string& idxB);
// text export of a plan and of the layout of the tensors it touches (plan_export.cpp)
void export_plan(const Context& ctx, const Plan& p, const char* path);

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

class Context {
public:
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Spaces spaces;
    bool spaces_set = false;
    std::map<int, std::unique_ptr<Tensor>> tensors;
    int next_handle = 1;
    std::string last_error;
    int64_t device_bytes = 0;
    int64_t peak_bytes = 0;
    bool host_only = false;            // device < 0: plan and account memory, launch nothing
    int64_t launches = 0;
    int precision = CCSD_PREC_FP64;
    int slices = 0;
    bool plan_refine = false;          // host-only plan of a split solve that may move to 4 slices
    int plan_threads = 8;              // host threads that plan the statements of an iteration
    double last_plan_flops = 0;        // algorithmic flops of the last ccsd_contract statement
    std::string last_plan_key;         // plan-cache key of the last ccsd_contract / ccsd_sum statement
    int split_routing = CCSD_SPLIT_ROUTE_AUTO;  // which contractions take the split kernel
    bool fp64_tiled_only = false;      // keep skinny FP64 products on the tiled kernel
    bool group_gemms = true;           // batch small block contractions of a statement into grouped launches
    int64_t split_launches = 0;        // split-BF16 GEMMs issued (host count)
    double* d_scalar = nullptr;        // device accumulator for dots
    kern::SplitWorkspace split_ws;     // scratch for split-BF16 GEMMs
    std::map<int64_t, kern::SlicedOperand> split_cache;   // sliced constant operands
    std::map<int64_t, int> split_owner;                    // cache key -> tensor handle
    int64_t split_cache_next = 1;
    kern::SlicedOperand ws_view[2];                        // workspace views of the current call
    double* merged_ws = nullptr;                           // dense products of merged launches
    int64_t merged_ws_elems = 0;
    std::vector<double*> merged_retired;                   // outgrown, kept until the context goes
    void build_merged(Plan& p, GemmRun& run, int first, int end, std::vector<char>& merged,
                      const std::function<std::pair<int, int64_t>(int, int64_t)>& block_of);
    void run_merged(Plan& p, MergedProduct& m, const std::string& label);
    void batch_merged_slicing(GemmRun& run, size_t launch0);
    int64_t merged_cache_bytes = 0;                        // reserved by merged products' cached slices
    void free_merged(MergedProduct& m);
    double* splitk_ws = nullptr;                           // FP64 split-K partials
    int64_t splitk_elems = 0;
    kern::SlicedOperand alloc_sliced(int rows, int K, int nslices, int kind);
    // slices per operand of the split path (3 unless set) and their kind
    int split_slices() const { return slices >= 3 ? slices : 3; }
    // slices of one split contraction: the context's count plus its autotuned delta
    int step_slices(const GemmStep& g) const { return std::max(3, split_slices() + g.slice_delta); }
    int slice_kind() const { return precision == CCSD_PREC_SPLIT_I8 ? kern::SLICE_INT8 : kern::SLICE_BF16; }
    bool split_precision() const { return precision == CCSD_PREC_SPLIT || precision == CCSD_PREC_SPLIT_I8; }
    void free_sliced(kern::SlicedOperand& s);
    void ensure_ws(kern::SlicedOperand& w, int rows, int K);
    void reserve_split(Plan& p);
    // drop the plan's cached slices and choose again for the current slice count (after a
    // 3 -> 4 slice switch), so that the cache is rebuilt within its budget largest-first
    void refresh_split(Plan& p);
    void drop_split_cache(GemmStep& g);
    std::map<std::string, std::unique_ptr<Plan>> plan_cache;

    // optional per-statement timing of GEMM steps with CUDA events on the stream
    bool profiling = false;
    struct ProfEntry {
        int64_t launches = 0;
        double flops = 0, ms = 0;
    };
    std::map<std::string, ProfEntry> profile;
    std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<double> pending_flops;
    std::vector<cudaEvent_t> event_pool;
    void collect_profile();
    std::pair<cudaEvent_t, cudaEvent_t> prof_begin();
    void prof_end(std::pair<cudaEvent_t, cudaEvent_t> ev, const std::string& label, double flops);

    Context(int device, cudaStream_t s);
    ~Context();

    Tensor& tensor(int h);
    int create_tensor(const std::string& name, const int nout[2], const int nin[2], int flags);
    // A tensor whose element (x_0..x_{n-1}) is the base tensor's element with x_p at base
    // position perm[p] (e.g. <ab||ci> = <ci||ab>); its blocks alias the base's storage.
    int create_view(const std::string& name, int base, const int nout[2], const int nin[2], const int* perm);
    void destroy_tensor(int h);
    void* dmalloc(size_t bytes);
    // Host -> device copy of plan tables and descriptors through a pinned staging arena:
    // stream-ordered, no implicit synchronisation (a copy from pageable memory waits for
    // the stream first); the arena is reused only after a stream synchronisation.
    void stage_h2d(void* dst, const void* src, size_t bytes);
    char* pin_buf = nullptr;
    size_t pin_cap = 0, pin_off = 0;
    void dfree(void* p, size_t bytes);

    // execute a plan on the stream (device tables uploaded lazily)
    void upload(Plan& p);
    void release(Plan& p);
    // scalar_out: host destination of the dot result (synchronises); dot_target: device
    // accumulator the dots add into instead of the context scalar (not zeroed here)
    void run(Plan& p, double* scalar_out = nullptr, double* dot_target = nullptr);
    void run_gemm(Plan& p, GemmStep& g);
    double* data_of(Plan& p, int h);
    void run_split_gemm(GemmStep& g, kern::GemmArgs& a);
    bool routes_split(const GemmStep& g) const;   // would run_gemm send g to the split kernel
    bool split_eligible(const GemmStep& g) const; // shape / operand rule of the split path
    kern::GemmArgs gemm_args(Plan& p, const GemmStep& g);
    RunSchedule& schedule(Plan& p);
    void build_run(Plan& p, RunSchedule& rs, int first, int end);
    void build_elementwise_run(Plan& p, RunSchedule& rs, int first, int end);
    void build_dot_run(Plan& p, RunSchedule& rs, int first, int end);
    void launch(Plan& p, const GemmLaunch& l, const std::string& label, double* dot_acc = nullptr);
    std::vector<int> constant_tensors;  // handles whose contents never change (sliced once)
    bool is_constant(int h) const;
};

Context* from_handle(ccsd_ctx c);

}  // namespace ccsd
