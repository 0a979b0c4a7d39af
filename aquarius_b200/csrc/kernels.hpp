// Launch wrappers for the engine's CUDA kernels (implemented in *.cu).
#pragma once
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

namespace ccsd {
namespace kern {

// C[Cm_v[m] + Cn_w[n]] += sign_vw * alpha * sum_k A[Am[m]+Ak[k]] * B[Bk[k]+Bn[n]]
struct GemmArgs {
    const double* A = nullptr;
    const double* B = nullptr;
    double* C = nullptr;
    int M = 0, N = 0, K = 0;
    double alpha = 0;
    const int64_t *Am = nullptr, *Ak = nullptr, *Bk = nullptr, *Bn = nullptr;
    const int64_t* Cm[2] = {nullptr, nullptr};
    const int64_t* Cn[2] = {nullptr, nullptr};
    int nvm = 1, nvn = 1;
    double vsign[4] = {1, 1, 1, 1};
    bool a_kcontig = false;   // consecutive k -> consecutive A addresses
    bool b_kcontig = false;   // consecutive k -> consecutive B addresses
    // split-K: partial products of ksplit K-ranges go to ws[z][m][n] (M*N*ksplit doubles)
    // and are folded in a fixed order before the scatter into C
    double* ws = nullptr;
    int64_t ws_elems = 0;
    // products with an extent <= 32 may take the skinny kernel (false: the tiled kernel only)
    bool skinny_ok = true;
    // Ak / Bk as arithmetic progressions (offset0 + k * step): no table loads on the
    // kernels' address path (the tables stay valid for the other users)
    bool ak_affine = false, bk_affine = false;
    int64_t ak0 = 0, ak_step = 0, bk0 = 0, bk_step = 0;
    // grouped launches with shared outputs: write the raw product to ws[m][n] (no alpha,
    // no scatter); a fold applies it to C
    bool partial_out = false;
    // split path: write the scaled product to ws[z][m][n] (dense, no alpha, no fold) for a
    // scatter by the caller (merged symmetry-blocked products)
    bool dense_out = false;
};

// Fold of dense partial products into C: with p = sum over z < ks of part[z*M*N + m*N + n]
// (the partials in order), C[Cm[a][m] + Cn[b][n]] += scale * vsign[a*nvn + b] * p for every
// variant (a, b); the problems of one group of output blocks in order.
struct FoldDesc {
    const double* part = nullptr;
    double* C = nullptr;
    const int64_t* Cm[2] = {nullptr, nullptr};
    const int64_t* Cn[2] = {nullptr, nullptr};
    int M = 0, N = 0, ks = 1, nvm = 1, nvn = 1;
    double vsign[4] = {1, 1, 1, 1};
    double scale = 0;
};
// one CTA per group: problems [group_start[g], group_start[g + 1]) of d, in order
void fold_groups(const FoldDesc* d, const int* group_start, int ngroups, cudaStream_t s);

// Skinny FP64 product: one small extent (<= 32) against a long operand L:
//   C[Cr_v[r] + Cs_w[s]] += sign_vw * alpha * sum_k L[Lr[r] + Lk[k]] * S[Sk[k] + Sn[s]]
struct SkinnyArgs {
    const double* L = nullptr;
    const double* S = nullptr;
    double* C = nullptr;
    const int64_t *Lr = nullptr, *Lk = nullptr, *Sk = nullptr, *Sn = nullptr;
    bool lk_affine = false, sk_affine = false;     // Lk / Sk as offset0 + k * step
    int64_t lk0 = 0, lk_step = 0, sk0 = 0, sk_step = 0;
    const int64_t* Cr[2] = {nullptr, nullptr};
    const int64_t* Cs[2] = {nullptr, nullptr};
    int R = 0, NS = 0, K = 0, nvr = 1, nvs = 1;
    double vsign[4] = {1, 1, 1, 1};   // [vr * nvs + vs]
    double alpha = 0;
    double* ws = nullptr;
    // grouped launches: nz K ranges per row tile; partial: every K range writes its raw
    // product to ws[z][r][s] for a fold (FoldDesc with ks = nz), even with nz = 1
    int nz = 1;
    bool partial = false;
};
// a contraction as a skinny product (the longer of M, N as the rows of L); *lk: L is
// contiguous along k
SkinnyArgs skinny_args(const GemmArgs& g, bool* lk);
// n-groups of 8 for a small extent (0: not a skinny product), and the row tiles of R rows
int skinny_groups(int M, int N);
int skinny_tiles(int R);
// many skinny products in one launch: tile_start[p] is the first of problem p's
// skinny_tiles(R) * nz CTAs; products writing C directly must have disjoint outputs
void skinny_grouped(const SkinnyArgs* d, const int* tile_start, int nprob, int tiles, int nt, bool lk,
                    cudaStream_t s);

// Short products: both extents <= 64 with (M/8) * (N/8) <= 16 fragments and a long K
// (F(mi) += <mn||ef> t(ef,in) per irrep block).  The CTAs of a problem split its K range
// (kper k each) and write their M x N partial products to part[cta][m][n]; a fold adds
// them (FoldDesc, ks = the problem's CTAs).  One launch covers every problem of one
// fragment shape, cta_start[p] being the first CTA of problem p.
struct ShortDesc {
    const double* A = nullptr;
    const double* B = nullptr;
    const int64_t *Am = nullptr, *Ak = nullptr, *Bk = nullptr, *Bn = nullptr;
    bool ak_affine = false, bk_affine = false;
    int64_t ak0 = 0, ak_step = 0, bk0 = 0, bk_step = 0;
    int M = 0, N = 0, K = 0, kper = 0;
    double* part = nullptr;
};
// fragment shape (m-fragments, n-fragments) of a short product, {0, 0} if it is not one
std::pair<int, int> short_shape(int M, int N);
// CTAs of a short product (its K range split in kper-multiples of 128)
int short_ctas(int K, int* kper);
void short_grouped(const ShortDesc* d, const int* cta_start, int nprob, int total_ctas, int mt, int nt,
                   cudaStream_t s);

// K-ranges the FP64 GEMM splits a contraction into (1 = none); ws needs ksplit*M*N doubles
int fp64_ksplit(int M, int N, int K, bool skinny_ok = true);

// native FP64 tensor-core (DMMA) GETT kernel
void gemm_fp64(const GemmArgs& g, cudaStream_t s);
// output tiles of the tiled FP64 kernel for an M x N product
int fp64_tiles(int M, int N);
// One launch of the tiled FP64 kernel over nprob problems (device array of GemmArgs, all
// with the given operand contiguity, no split-K, pairwise disjoint outputs); tile_start
// (device, nprob entries) holds each problem's first tile.
void gemm_fp64_grouped(const GemmArgs* probs, const int* tile_start, int nprob, int total_tiles, bool a_kcontig,
                       bool b_kcontig, cudaStream_t s);

// ---- split (Ozaki-style) path ----------------------------------------------------
// Slice kinds: BF16 slices of 8 significant bits (3 or 4 per operand, FP32 tensor
// accumulation) or INT8 slices of 7 bits (3, 4 or 5 per operand, exact INT32 tensor
// accumulation at twice the BF16 rate).
enum SliceKind { SLICE_BF16 = 0, SLICE_INT8 = 1 };
inline int slice_elem_bytes(int kind) { return kind == SLICE_INT8 ? 1 : 2; }
inline bool slice_scheme_ok(int kind, int ns) {
    return kind == SLICE_INT8 ? (ns >= 3 && ns <= 5) : (ns == 3 || ns == 4);
}

// An operand sliced for the tcgen05 GEMM: rows x kpad values per slice, K-major, row
// scale 2^e per row.  rows is padded to a multiple of 128, kpad to one 128-byte k-block
// (64 BF16 or 128 INT8 values).
struct SlicedOperand {
    uint8_t* data = nullptr;    // [nslices][rows][kpad] elements of the kind
    double* scale = nullptr;    // [rows]  value = scale * sum_t w_t s_t
    double* rowmax = nullptr;   // [rows]  scratch of the slicing pass
    int rows = 0, kpad = 0, nslices = 0, kind = SLICE_BF16;
    int64_t bytes = 0;          // allocated slice bytes (capacity of a workspace)
};

struct SplitWorkspace {
    SlicedOperand a, b;          // per-call slices of non-constant operands
};

// number of bf16 slices of the split path
constexpr int kDefaultSlices = 3;
int split_rows_pad(int rows);
int split_k_pad(int k, int kind);
// slice bytes of a rows x K operand in a scheme (without the row scales)
inline int64_t split_slice_bytes(int rows, int K, int ns, int kind) {
    return (int64_t)ns * split_rows_pad(rows) * split_k_pad(K, kind) * slice_elem_bytes(kind);
}

// slice rows of X(r,k) = X[R[r] + Kt[k]] (r < nrows, k < K) into `out` (allocated by caller
// with out.rows >= nrows padded, out.kpad >= K padded; out.kind and out.nslices say how)
void slice_rows(const double* X, const int64_t* R, const int64_t* Kt, int nrows, int K, bool kcontig,
                SlicedOperand& out, cudaStream_t s);
// tcgen05 GEMM over slices; epilogue scatters into C like gemm_fp64.  ks > 1 splits K
// into ks ranges whose partials go to g.ws (ks * M * N doubles) and are folded into C.
void gemm_split(const SlicedOperand& a, const SlicedOperand& b, int M, int N, int K,
                const GemmArgs& g, cudaStream_t s, int ks = 1);
// K-ranges for a split GEMM: enough CTAs for about two waves when the output has few
// tiles (1 = none)
int split_ksplit(int M, int N, int K, int nslices = 3, int kind = SLICE_BF16);
// alpha * sum_z ws[z][m][n] scattered into every destination variant of g (fixed order)
void splitk_fold(const GemmArgs& g, int ks, cudaStream_t s);

// Merged products of a symmetry-blocked statement: the block products of one irrep class
// form one dense GEMM.  Its operands are rectangles (a block product's rows x its k range)
// placed at (row0, k0) of a merged operand; its result goes to a dense workspace and is
// scattered into the C blocks rectangle by rectangle.
struct RectDesc {
    const double* X = nullptr;     // storage the rectangle's offsets index
    const int64_t* R = nullptr;    // row offsets (nrows)
    const int64_t* Kt = nullptr;   // k offsets (nk)
    int nrows = 0, nk = 0;
    int row0 = 0, k0 = 0;          // position in the merged operand
    int kc = 0;                    // neighbouring k adjacent in memory (lanes along k)
    int tiles_r = 0;               // 32-row tiles of the rectangle
    double mul = 1.0;              // factor of the rectangle's values (its product's coefficient
                                   // relative to the class's, folded into the B operand)
    // batched slicing: the rectangle's own merged operand (null: the launch's operand)
    uint8_t* out = nullptr;        // [5 slices][rows_p][kpad], zero outside the rectangles
    double* scale = nullptr;       // [rows_p]
    unsigned long long* rowmax = nullptr;   // [rows_p]
    int rows_p = 0, kpad = 0;
};
// row maxima over all rectangles of a row, then INT8 slices of every rectangle into out
// (its rows, scales and slices zeroed first); tile_start[i] = first 32 x 64 tile of
// rectangle i, ntiles in all
void rect_slice(const RectDesc* d, const int64_t* tile_start, int n, int64_t ntiles, int ns, SlicedOperand& out,
                cudaStream_t s);
// the rectangles of many merged operands (each with its own destination) in one rowmax
// and one slice launch; rowmax_arena (bytes) holds every destination's row maxima
void rect_slice_batched(const RectDesc* d, const int64_t* tile_start, int n, int64_t ntiles, int ns,
                        void* rowmax_arena, size_t rowmax_bytes, cudaStream_t s);
struct ScatterDesc {
    double* C = nullptr;
    const int64_t* Cm[2] = {nullptr, nullptr};
    const int64_t* Cn[2] = {nullptr, nullptr};
    int nvm = 1, nvn = 1;
    double vsign[4] = {1, 1, 1, 1};
    double alpha = 0;
    int nrows = 0, ncols = 0, row0 = 0, col0 = 0;
};
// C += alpha * sum_z ws[z] over each rectangle (chunks of kBatchChunk elements)
void rect_scatter(const ScatterDesc* d, const int64_t* chunk_start, int n, int64_t chunks, const double* ws, int ldn,
                  int64_t zstride, int ks, cudaStream_t s);
bool split_supported();
// nonzero if a split-GEMM wait expired (1..4 = which wait); reset clears it
int split_error(bool reset);

// ---- elementwise / reductions ----------------------------------------------------
struct StridedArgs {
    int ndim = 0;
    int64_t len[8];
    int64_t sA[8], sB[8];
    int64_t total = 1;
};
// C[offC + sum idx*sB] += alpha * A[offA + sum idx*sA]
void sum_strided(const double* A, double* C, const StridedArgs& a, double alpha, cudaStream_t s);
// out[0] += alpha * sum A[..]*B[..]
void dot_strided(const double* A, const double* B, const StridedArgs& a, double alpha, double* out,
                 cudaStream_t s);
void scale(double* X, int64_t n, double beta, cudaStream_t s);
void fill(double* X, int64_t n, double val, cudaStream_t s);
// max |x| (p=0), sum |x| (p=1) or sum x^2 (p=2) of n elements, accumulated into out[0]
// with weight w (p=1,2) or max (p=0)
void norm_accum(const double* X, int64_t n, int p, double w, double* out, cudaStream_t s);
// out = alpha*x + beta*out
void axpby(const double* x, double* out, int64_t n, double alpha, double beta, cudaStream_t s);

// Jacobi weight of one block: x /= (sum_p d_p[idx_p] + shift), 0 if |.| < 1e-4
struct WeightArgs {
    int ndim = 0;
    int64_t len[8];
    const double* d[8];
    int64_t total = 1;
};
void weight_block(double* X, const WeightArgs& w, double shift, cudaStream_t s);

// key/value scatter: X[keys[i]] = beta*X[keys[i]] + alpha*vals[i]
void kv_write(double* X, const int64_t* keys, const double* vals, int64_t n, double alpha, double beta,
              cudaStream_t s);
void kv_read(const double* X, const int64_t* keys, double* vals, int64_t n, cudaStream_t s);

// ---- fused CCSD update / DIIS -------------------------------------------------------
// z = w * z_raw / den (den from per-position denominators), t += z, track max|z|;
// blocks described by WeightArgs; results accumulated into red[0] (max)
void update_block(double* Z, double* T, const WeightArgs& w, double* red_max, cudaStream_t s);

// batched dot: out[j] += w * sum x[i]*ys[j][i], j < ny  (ys: device array of pointers)
void dot_batch(const double* x, const double* const* ys, int ny, int64_t n, double w, double* out,
               cudaStream_t s);
// out[i] = sum_j c[j] * xs[j][i]  (c on device); i < n1 goes to out1, the rest to out2
void lincomb(double* out1, int64_t n1, double* out2, int64_t n2, const double* const* xs, const double* c, int nx,
             cudaStream_t s);

// ---- device-resident DIIS (src/convergence/diis.hpp:70-227) -----------------------------
// state[0] = slot of the newest vector, state[1] = stored vectors, state[2] = start counter,
// state[3] = singular flag.  The ring keeps `order` vectors; slot (head - k) mod order holds
// the vector of k iterations ago.
void diis_advance(int* state, int order, cudaStream_t s);
// xs[head] = [t1 | t2], dxs[head] = [z1 | z2]
void diis_store(const int* state, const double* const* xs, const double* const* dxs, const double* t1, int64_t n1,
                const double* t2, int64_t n2, const double* z1, const double* z2, cudaStream_t s);
// dots[j] += w * <dxs[head][off:off+len], dxs[j][off:off+len]>,  j < order
void diis_dots(const int* state, const double* const* dxs, int order, int64_t off, int64_t len, double w,
               double* dots, cudaStream_t s);
// update the error matrix with the new row, solve the bordered system and write the
// coefficients by slot into c (unit vector at head when no extrapolation happens)
void diis_solve(int* state, double* e, double* c, const double* dots, int order, cudaStream_t s);
// standalone DIIS over caller tensors: one (x, dx) piece into the head slot at `off`
void diis_store_segment(const int* state, const double* const* xs, const double* const* dxs, int64_t off,
                        const double* x, const double* dx, int64_t len, cudaStream_t s);
// out[i] = sum_j c[j] * xs[j][off + i], i < len
void lincomb_segment(double* out, int64_t len, const double* const* xs, int64_t off, const double* c, int nx,
                     cudaStream_t s);
// the damping branch of diis.hpp:155-161 on the stored newest x (after diis_solve)
void diis_damp(const int* state, const double* const* xs, int order, int64_t len, double damping, cudaStream_t s);

// Pack <ab||cd> = J - K for canonical pairs of a packed block, a in [a0,a1):
//   J = tJ[a-a0, c, b, d] = (ac|bd),  K = tK[a-a0, d, b, c] = (ad|bc)
// kind 1: triangle (x<y, equal irreps), kind 2: full rectangle.  The (a,b) pair has
// stride 1, the (c,d) pair stride `scd`.
void pack_vvvv(double* V, int kind_ab, int kind_cd, int n0, int n1, int n2, int n3, int64_t scd, const double* tJ,
               const double* tK, int a0, int a1, bool J, bool K, cudaStream_t s);

// One block of Tau: tau[a,b,i,j] = t2[a,b,i,j] + t1ai[a,i] t1bj[b,j] - t1aj[a,j] t1bi[b,i]
// (blocks first index fastest; a T1 block [x,y] has leading dimension len of x; a null
// pair drops its term)
struct TauArgs {
    double* tau = nullptr;
    const double* t2 = nullptr;
    const double *t1ai = nullptr, *t1bj = nullptr, *t1aj = nullptr, *t1bi = nullptr;
    int64_t len[4] = {0, 0, 0, 0};
};
void tau_block(const TauArgs& a, cudaStream_t s);
// closed-shell two-electron Fock part from dense (pq|rs) (last index fastest):
// F[p*n + q] = sum_{i < nocc} 2 (pq|ii) - (pi|iq)
void closed_shell_jk(const double* eri, int n, int nocc, double* F, cudaStream_t s);
// every block of Tau in one launch: chunks of kBatchChunk elements, chunk_start[p] the
// first chunk of block p (device arrays)
void tau_batched(const TauArgs* d, const int64_t* chunk_start, int n, int64_t chunks, cudaStream_t s);

// Jacobi update of many blocks in one launch: z = z / den, t += z, red_max = max |z|
struct UpdateDesc {
    double* Z = nullptr;
    double* T = nullptr;
    WeightArgs w;
};
void update_batched(const UpdateDesc* d, const int64_t* chunk_start, int n, int64_t chunks, double* red_max,
                    cudaStream_t s);

// Dots of many strided blocks in one launch: part[c] = partial sum of chunk c, then one
// CTA adds sum_c part[c] (fixed order) to out[0]
struct DotDesc {
    const double* A = nullptr;
    const double* B = nullptr;
    int ndim = 0;
    int64_t len[8], sA[8], sB[8];
    int64_t total = 0;
    double alpha = 0;
    int fast = 0;                      // multiply-shift index split, as SumDesc
    uint32_t dmul[8], dshr[8];
};
// fill the multiply-shift divisors of a sum / dot descriptor (fast = 0 when an index may
// reach 2^31)
void plan_divisors(const int64_t* len, int ndim, int64_t total, int& fast, uint32_t* dmul, uint32_t* dshr);
void dot_batched(const DotDesc* d, const int64_t* chunk_start, int n, int64_t chunks, double* part, double* out,
                 cudaStream_t s);

// Gather of a dense spatial (pq|rs) array (n^4, last index fastest) into a block:
//   C[off + sum_p st[p] x_p] += sign * eri[((g0 n + g1) n + g2) n + g3],
//   g_k = g[pos[k]][x_pos[k]]
// with g[p] the orbital index of every x on position p (device tables).  Distinct x
// must map to distinct elements of C.
struct EriGatherArgs {
    double* C = nullptr;
    int64_t off = 0;
    int len[4] = {1, 1, 1, 1};
    int64_t st[4] = {0, 0, 0, 0};
    const int* g[4] = {nullptr, nullptr, nullptr, nullptr};
    int pos[4] = {0, 1, 2, 3};
    int64_t n = 0;
    double sign = 1.0;
};
void eri_gather(const EriGatherArgs& a, const double* eri, cudaStream_t s);

int64_t launch_count();
void reset_launch_count();
// free the reduction scratch kept for a stream (before the stream is destroyed)
void release_stream_buffers(cudaStream_t s);

// Batched permuted sums C[perm] += alpha * A and block scalings, one launch each: the
// problems (device arrays) must write pairwise disjoint elements; chunk_start[p] is the
// first 2048-element chunk of problem p.
constexpr int kBatchChunk = 2048;
struct SumDesc {
    const double* A = nullptr;
    double* C = nullptr;
    double alpha = 0;
    int ndim = 0;
    int64_t len[8], sA[8], sC[8];
    int64_t total = 0;
    // permuted sums whose fastest A and C positions differ go through 32 x 32 shared-memory
    // tiles over those two positions (coalesced reads of A and writes of C); a chunk is
    // two tiles
    int tiled = 0, p0 = 0, pc = 0;
    int64_t ntiles = 0;
    // every index below 2^31: the element index splits into positions by multiply-shift
    // (x / len = (umulhi(x, mul) + x) >> shr) instead of 64-bit divisions
    int fast = 0;
    uint32_t dmul[8], dshr[8];
};
// chunks of kBatchChunk elements (or two 32 x 32 tiles) a sum descriptor takes
inline int64_t sum_chunks(const SumDesc& d) {
    return d.tiled ? (d.ntiles + 1) / 2 : (d.total + kBatchChunk - 1) / kBatchChunk;
}
// fill the tiling fields of a descriptor (after len / sA / sC / total)
void sum_plan_tiles(SumDesc& d);
struct ScaleDesc {
    double* X = nullptr;
    int64_t n = 0;
    double beta = 1;   // 0: zero-fill
};
void sum_batched(const SumDesc* d, const int64_t* chunk_start, int n, int64_t chunks, cudaStream_t s);
void scale_batched(const ScaleDesc* d, const int64_t* chunk_start, int n, int64_t chunks, cudaStream_t s);

}  // namespace kern
}  // namespace ccsd
