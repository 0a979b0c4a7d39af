// Native-FP64 kernels: the DMMA gather-GEMM ("plain path" contraction layer) and the
// HBM-bound elementwise / reduction kernels of the iteration.
//
// The GEMM computes, for one planned block contraction,
//   C[Cm_v[m] + Cn_w[n]] += s_vw * alpha * sum_k A[Am[m]+Ak[k]] * B[Bk[k]+Bn[n]]
// i.e. a GEMM whose operands are gathered straight from the stored tensor blocks
// through per-dimension offset tables (no separate transpose pass), and whose
// epilogue scatters into the output block, once per antisymmetric image.
#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <set>
#include <utility>
#include <algorithm>
#include <stdexcept>
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace ccsd {
namespace kern {

std::atomic<int64_t> g_launches{0};
int64_t launch_count() { return g_launches.load(); }
void reset_launch_count() { g_launches = 0; }
#define COUNT_LAUNCH() (g_launches++)

// dynamic shared memory above 48 KiB must be opted into once per kernel and device;
// contexts on several host threads may launch the same kernel first
void set_smem_once(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.insert({kernel, dev}).second) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// ---------------------------------------------------------------------------
// FP64 DMMA gather-GEMM
// ---------------------------------------------------------------------------
namespace {

constexpr int BM = 128, BN = 64, BK = 16, STAGES = 3, THREADS = 256;
constexpr int LDMK = BM + 8;   // A stored [k][m]
constexpr int LDNK = BN + 8;   // B stored [k][n]
constexpr int LDK = BK + 4;    // operands stored [m][k] / [n][k]

template <bool AK, bool BK_>
struct Smem {
    static constexpr int a_elems = AK ? BM * LDK : BK * LDMK;
    static constexpr int b_elems = BK_ ? BN * LDK : BK * LDNK;
    static constexpr size_t bytes = (size_t)STAGES * (a_elems + b_elems) * sizeof(double) + (BM + BN) * sizeof(int64_t);
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One BM x BN output tile of one problem, K-range kz of nz (split-K writes raw partials
// to g.ws[kz]).  smem_raw: the dynamic shared memory of Smem<AK, BKc>.
template <bool AK, bool BKc>
__device__ __forceinline__ void fp64_tile(const GemmArgs& g, const int m0, const int n0, const int kz, const int nz,
                                          unsigned char* smem_raw) {
    using S = Smem<AK, BKc>;
    double* As = reinterpret_cast<double*>(smem_raw);
    double* Bs = As + STAGES * S::a_elems;
    int64_t* sAm = reinterpret_cast<int64_t*>(Bs + STAGES * S::b_elems);
    int64_t* sBn = sAm + BM;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;

    for (int i = tid; i < BM; i += THREADS) sAm[i] = (m0 + i < g.M) ? g.Am[m0 + i] : 0;
    for (int i = tid; i < BN; i += THREADS) sBn[i] = (n0 + i < g.N) ? g.Bn[n0 + i] : 0;
    __syncthreads();

    // this CTA's K-range (split-K: range kz of nz)
    const int ktiles_all = (g.K + BK - 1) / BK;
    const int per_split = (ktiles_all + nz - 1) / nz;
    const int kt0 = kz * per_split;
    const int ktiles = max(0, min(ktiles_all, kt0 + per_split) - kt0);

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * BK;
        double* as = As + stage * S::a_elems;
        double* bs = Bs + stage * S::b_elems;
        // A tile: BM x BK
#pragma unroll
        for (int i = 0; i < (BM * BK) / THREADS; i++) {
            int e = tid + i * THREADS;
            int m, k;
            if (AK) { k = e % BK; m = e / BK; }
            else    { m = e % BM; k = e / BM; }
            bool ok = (m0 + m < g.M) && (k0 + k < g.K);
            const double* src =
                ok ? g.A + sAm[m] + (g.ak_affine ? g.ak0 + g.ak_step * (k0 + k) : __ldg(g.Ak + k0 + k)) : g.A;
            double* dst = AK ? as + m * LDK + k : as + k * LDMK + m;
            cp_async8(dst, src, ok);
        }
        // B tile: BK x BN
#pragma unroll
        for (int i = 0; i < (BN * BK) / THREADS; i++) {
            int e = tid + i * THREADS;
            int n, k;
            if (BKc) { k = e % BK; n = e / BK; }
            else     { n = e % BN; k = e / BN; }
            bool ok = (n0 + n < g.N) && (k0 + k < g.K);
            const double* src =
                ok ? g.B + sBn[n] + (g.bk_affine ? g.bk0 + g.bk_step * (k0 + k) : __ldg(g.Bk + k0 + k)) : g.B;
            double* dst = BKc ? bs + n * LDK + k : bs + k * LDNK + n;
            cp_async8(dst, src, ok);
        }
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < ktiles) load_stage(s, kt0 + s);
        cp_commit();
    }

    for (int kt = 0; kt < ktiles; kt++) {
        cp_wait<STAGES - 2>();
        __syncthreads();
        {
            int nk = kt + STAGES - 1;
            if (nk < ktiles) load_stage(nk % STAGES, kt0 + nk);
            cp_commit();
        }
        const double* as = As + (kt % STAGES) * S::a_elems;
        const double* bs = Bs + (kt % STAGES) * S::b_elems;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double af[4], bf[4];
            const int kr = kk + (lane & 3);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                int m = wm + i * 8 + (lane >> 2);
                af[i] = AK ? as[m * LDK + kr] : as[kr * LDMK + m];
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                int n = wn + j * 8 + (lane >> 2);
                bf[j] = BKc ? bs[n * LDK + kr] : bs[kr * LDNK + n];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    cp_wait<0>();

    if (nz > 1 || g.partial_out) {
        // split-K (or a shared-output group): raw partial sums, folded by splitk_fold_kernel
        // (fold_groups_kernel)
        double* wz = g.ws + (int64_t)kz * g.M * g.N;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int m = m0 + wm + i * 8 + (lane >> 2);
            if (m >= g.M) continue;
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    int n = n0 + wn + j * 8 + 2 * (lane & 3) + h;
                    if (n < g.N) wz[(int64_t)m * g.N + n] = acc[i][j][h];
                }
        }
        return;
    }

    if (g.nvm == 1 && g.nvn == 1) {
        // one destination per element: the 8 read-modify-writes of a row group are
        // issued as 8 reads, then 8 writes (overlapped instead of one by one)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int m = m0 + wm + i * 8 + (lane >> 2);
            if (m >= g.M) continue;
            const int64_t cm = g.Cm[0][m];
            const double sc = g.alpha * g.vsign[0];
            int64_t off[8];
            double old[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int n = n0 + wn + (t >> 1) * 8 + 2 * (lane & 3) + (t & 1);
                off[t] = n < g.N ? cm + g.Cn[0][n] : -1;
            }
#pragma unroll
            for (int t = 0; t < 8; t++) old[t] = off[t] >= 0 ? g.C[off[t]] : 0.0;
#pragma unroll
            for (int t = 0; t < 8; t++)
                if (off[t] >= 0) g.C[off[t]] = old[t] + sc * acc[i][t >> 1][t & 1];
        }
        return;
    }
    // epilogue: scatter to every destination variant
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int m = m0 + wm + i * 8 + (lane >> 2);
        if (m >= g.M) continue;
        int64_t cm[2];
        cm[0] = g.Cm[0][m];
        cm[1] = g.nvm > 1 ? g.Cm[1][m] : 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int n = n0 + wn + j * 8 + 2 * (lane & 3) + h;
                if (n >= g.N) continue;
                double v = g.alpha * acc[i][j][h];
                for (int a = 0; a < g.nvm; a++)
                    for (int b = 0; b < g.nvn; b++) {
                        double* dst = g.C + cm[a] + g.Cn[b][n];
                        *dst += g.vsign[a * g.nvn + b] * v;
                    }
            }
        }
    }
}

template <bool AK, bool BKc>
__global__ void __launch_bounds__(THREADS, 1) gemm_fp64_kernel(GemmArgs g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    fp64_tile<AK, BKc>(g, blockIdx.y * BM, blockIdx.x * BN, blockIdx.z, gridDim.z, smem_raw);
}

// Grouped launch: one CTA per output tile of any of nprob problems whose outputs are
// pairwise disjoint; tile_start[p] is the first tile of problem p.
template <bool AK, bool BKc>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_fp64_grouped_kernel(const GemmArgs* __restrict__ probs, const int* __restrict__ tile_start, int nprob) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ GemmArgs sg;
    __shared__ int sp;
    const int t = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile_start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        sp = lo;
        sg = probs[lo];
    }
    __syncthreads();
    const int local = t - tile_start[sp];
    const int tn = (sg.N + BN - 1) / BN;
    fp64_tile<AK, BKc>(sg, (local / tn) * BM, (local % tn) * BN, 0, 1, smem_raw);
}

// shared-output groups: each CTA folds the partial products of one group of output blocks,
// its problems one after another and each problem's partials in order (fixed order)
__global__ void fold_groups_kernel(const FoldDesc* __restrict__ d, const int* __restrict__ gstart) {
    const int g = blockIdx.x;
    for (int p = gstart[g]; p < gstart[g + 1]; p++) {
        const FoldDesc f = d[p];
        const int64_t mn = (int64_t)f.M * f.N;
        for (int64_t l = threadIdx.x; l < mn; l += blockDim.x) {
            double s = 0.0;
            for (int z = 0; z < f.ks; z++) s += f.part[z * mn + l];
            const int m = (int)(l / f.N), n = (int)(l % f.N);
            const double v = f.scale * s;
            for (int a = 0; a < f.nvm; a++)
                for (int b = 0; b < f.nvn; b++) f.C[f.Cm[a][m] + f.Cn[b][n]] += f.vsign[a * f.nvn + b] * v;
        }
        __syncthreads();
    }
}

// fold split-K partials in a fixed order and scatter alpha * sum into every variant
__global__ void splitk_fold_kernel(GemmArgs g, int ks) {
    const int64_t mn = (int64_t)g.M * g.N;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < mn; l += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < ks; z++) s += g.ws[z * mn + l];
        const int m = (int)(l / g.N), n = (int)(l % g.N);
        const double v = g.alpha * s;
        for (int a = 0; a < g.nvm; a++)
            for (int b = 0; b < g.nvn; b++) g.C[g.Cm[a][m] + g.Cn[b][n]] += g.vsign[a * g.nvn + b] * v;
    }
}

// ---------------------------------------------------------------------------
// Skinny FP64 product: one small extent (<= 32) against a long operand.
//   C[Cr_v[r] + Cs_w[s]] += sign_vw * alpha * sum_k L[Lr[r] + Lk[k]] * S[Sk[k] + Sn[s]]
// A CTA owns SK_TM rows of the long operand L and one K range.  L streams through shared
// memory in SK_TM x SK_KC tiles (cp.async, SK_STAGES stages, 16-byte copies where two
// neighbouring elements are contiguous and aligned; coalesced along whichever of r / k is
// contiguous); the small operand's SK_KC x 8*NT tile sits beside it.  The k offsets of
// both operands for a stage are staged in shared memory one stage ahead, so no copy
// waits on a table load.  Each warp computes 32 rows x 8*NT columns on the FP64 tensor
// cores (mma.m8n8k4: 4 x NT tiles per warp, 32 accumulators per thread), so the issue
// slots go to the loads and not to one FMA per element pair.  A short long-extent splits
// K over gridDim.z into ws[z][r][s], folded in a fixed order.
// ---------------------------------------------------------------------------
constexpr int SK_THREADS = 256, SK_STAGES = 4, SK_TM = 256, SK_KC = 8;

template <int NT, bool LK>
struct SkinnyShape {
    static constexpr int MT = 4;                          // m-tiles of 8 rows per warp (8 warps x 32 rows)
    static constexpr int LDA = SK_TM + 8;                 // [k][r] (r contiguous): 8 mod 16 doubles
    static constexpr int A_ELEMS = LK ? SK_TM * SK_KC : SK_KC * LDA;
    static constexpr int LDB = 8 * NT + (NT > 1 ? 8 : 0); // [k][s]: 8 mod 16 doubles
    static constexpr int B_ELEMS = SK_KC * LDB;
    static constexpr size_t bytes = (size_t)SK_STAGES * (A_ELEMS + B_ELEMS) * sizeof(double) +
                                    (SK_TM + 8 * NT + 2 * SK_STAGES * SK_KC) * sizeof(int64_t);
};

// [r][k] tiles (k contiguous, 8 per row): k XOR 4 on every other pair of rows, so that the
// eight rows x four k of an A fragment fall on 16 different double banks
__device__ __forceinline__ int lk_index(int r, int k) { return r * SK_KC + (k ^ (((r >> 1) & 1) << 2)); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

// one CTA: rows [rtile * SK_TM, +SK_TM) of the long operand over K range z of nz
template <int NT, bool LK>
__device__ __forceinline__ void skinny_body(const SkinnyArgs& g, int rtile, int z, int nz, unsigned char* smem_raw) {
    using Sh = SkinnyShape<NT, LK>;
    double* As = reinterpret_cast<double*>(smem_raw);
    double* Bs = As + SK_STAGES * Sh::A_ELEMS;
    int64_t* sLr = reinterpret_cast<int64_t*>(Bs + SK_STAGES * Sh::B_ELEMS);
    int64_t* sSn = sLr + SK_TM;
    int64_t* sLk = sSn + 8 * NT;                 // [stage][k]: offsets of L, -1 past K
    int64_t* sSk = sLk + SK_STAGES * SK_KC;      // [stage][k]: offsets of S

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = rtile * SK_TM;
    for (int i = tid; i < SK_TM; i += SK_THREADS) sLr[i] = (r0 + i < g.R) ? g.Lr[r0 + i] : -1;
    for (int i = tid; i < 8 * NT; i += SK_THREADS) sSn[i] = (i < g.NS) ? g.Sn[i] : -1;

    const int kchunks_all = (g.K + SK_KC - 1) / SK_KC;
    const int per_split = (kchunks_all + nz - 1) / nz;
    const int kc0 = z * per_split;
    const int kchunks = max(0, min(kchunks_all, kc0 + per_split) - kc0);

    // the k offsets of chunk c (relative to this CTA's range) into table slot c % stages
    auto load_table = [&](int c) {
        if (tid < 2 * SK_KC && c < kchunks) {
            const int k = (kc0 + c) * SK_KC + (tid % SK_KC);
            int64_t v = -1;
            if (k < g.K) {
                if (tid < SK_KC) v = g.lk_affine ? g.lk0 + g.lk_step * k : __ldg(g.Lk + k);
                else v = g.sk_affine ? g.sk0 + g.sk_step * k : __ldg(g.Sk + k);
            }
            (tid < SK_KC ? sLk : sSk)[(c % SK_STAGES) * SK_KC + (tid % SK_KC)] = v;
        }
    };
    auto load_stage = [&](int c) {
        const int st = c % SK_STAGES;
        double* as = As + st * Sh::A_ELEMS;
        double* bs = Bs + st * Sh::B_ELEMS;
        const int64_t* lk = sLk + st * SK_KC;
        const int64_t* sk = sSk + st * SK_KC;
        // the long operand in pairs of neighbours (rows for [k][r], k for [r][k])
#pragma unroll
        for (int i = 0; i < (SK_TM * SK_KC / 2) / SK_THREADS; i++) {
            const int e = tid + i * SK_THREADS;
            int r, k, r1, k1;
            double *d0, *d1;
            if (LK) {
                r = e / (SK_KC / 2);
                k = 2 * (e % (SK_KC / 2));
                r1 = r;
                k1 = k + 1;
                d0 = as + lk_index(r, k);
                d1 = d0 + 1;
            } else {
                k = e / (SK_TM / 2);
                r = 2 * (e % (SK_TM / 2));
                r1 = r + 1;
                k1 = k;
                d0 = as + k * Sh::LDA + r;
                d1 = d0 + 1;
            }
            const int64_t o0r = sLr[r], o1r = sLr[r1], o0k = lk[k], o1k = lk[k1];
            const bool ok0 = o0r >= 0 && o0k >= 0, ok1 = o1r >= 0 && o1k >= 0;
            const int64_t o0 = o0r + o0k, o1 = o1r + o1k;
            if (ok0 && ok1 && o1 == o0 + 1 && !(o0 & 1) && !((reinterpret_cast<uintptr_t>(g.L)) & 15)) {
                cp_async16(d0, g.L + o0);
            } else {
                cp_async8(d0, ok0 ? g.L + o0 : g.L, ok0);
                cp_async8(d1, ok1 ? g.L + o1 : g.L, ok1);
            }
        }
        for (int e = tid; e < SK_KC * 8 * NT; e += SK_THREADS) {
            const int sidx = e % (8 * NT), k = e / (8 * NT);
            const bool ok = sSn[sidx] >= 0 && sk[k] >= 0;
            cp_async8(bs + k * Sh::LDB + sidx, ok ? g.S + sSn[sidx] + sk[k] : g.S, ok);
        }
    };

    double acc[Sh::MT][NT][2];
#pragma unroll
    for (int i = 0; i < Sh::MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    for (int c = 0; c < SK_STAGES; c++) load_table(c);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < SK_STAGES - 1; c++) {
        if (c < kchunks) load_stage(c);
        cp_commit();
    }
    const int wr = warp * 8 * Sh::MT;            // first row of this warp in the tile
    const int fr = lane >> 2, fk = lane & 3;      // fragment row / k of this lane
    for (int c = 0; c < kchunks; c++) {
        cp_wait<SK_STAGES - 2>();
        __syncthreads();
        {
            const int nc = c + SK_STAGES - 1;
            if (nc < kchunks) load_stage(nc);
            cp_commit();
            load_table(c + SK_STAGES);           // the slot of chunk c, whose copies are issued
        }
        const double* as = As + (c % SK_STAGES) * Sh::A_ELEMS;
        const double* bs = Bs + (c % SK_STAGES) * Sh::B_ELEMS;
#pragma unroll
        for (int ks = 0; ks < SK_KC / 4; ks++) {
            double a[Sh::MT], b[NT];
            const int k = 4 * ks + fk;
#pragma unroll
            for (int i = 0; i < Sh::MT; i++) {
                const int r = wr + 8 * i + fr;
                a[i] = LK ? as[lk_index(r, k)] : as[k * Sh::LDA + r];
            }
#pragma unroll
            for (int j = 0; j < NT; j++) b[j] = bs[k * Sh::LDB + 8 * j + fr];
#pragma unroll
            for (int i = 0; i < Sh::MT; i++)
#pragma unroll
                for (int j = 0; j < NT; j++) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_wait<0>();

    // lane holds rows wr + 8i + fr, columns 8j + 2 fk + {0, 1}
    if (nz > 1 || g.partial) {
        double* wz = g.ws + (int64_t)z * g.R * g.NS;
#pragma unroll
        for (int i = 0; i < Sh::MT; i++) {
            const int r = r0 + wr + 8 * i + fr;
            if (r >= g.R) continue;
#pragma unroll
            for (int j = 0; j < NT; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int sidx = 8 * j + 2 * fk + h;
                    if (sidx < g.NS) wz[(int64_t)r * g.NS + sidx] = acc[i][j][h];
                }
        }
        return;
    }
    if (g.nvr == 1 && g.nvs == 1) {
        // one destination per element: the reads of a row batch first, then the writes
        const double sc = g.alpha * g.vsign[0];
#pragma unroll
        for (int i = 0; i < Sh::MT; i++) {
            const int r = r0 + wr + 8 * i + fr;
            if (r >= g.R) continue;
            const int64_t cr = g.Cr[0][r];
            int64_t off[2 * NT];
            double old[2 * NT];
#pragma unroll
            for (int j = 0; j < NT; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int sidx = 8 * j + 2 * fk + h;
                    off[2 * j + h] = sidx < g.NS ? cr + g.Cs[0][sidx] : -1;
                }
#pragma unroll
            for (int q = 0; q < 2 * NT; q++) old[q] = off[q] >= 0 ? g.C[off[q]] : 0.0;
#pragma unroll
            for (int j = 0; j < NT; j++)
#pragma unroll
                for (int h = 0; h < 2; h++)
                    if (off[2 * j + h] >= 0) g.C[off[2 * j + h]] = old[2 * j + h] + sc * acc[i][j][h];
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < Sh::MT; i++) {
        const int r = r0 + wr + 8 * i + fr;
        if (r >= g.R) continue;
        int64_t cr[2];
        cr[0] = g.Cr[0][r];
        cr[1] = g.nvr > 1 ? g.Cr[1][r] : 0;
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int sidx = 8 * j + 2 * fk + h;
                if (sidx >= g.NS) continue;
                const double v = g.alpha * acc[i][j][h];
                for (int a = 0; a < g.nvr; a++)
                    for (int b = 0; b < g.nvs; b++) g.C[cr[a] + g.Cs[b][sidx]] += g.vsign[a * g.nvs + b] * v;
            }
    }
}

// two CTAs per SM (about 80 KB of shared memory each): 16 warps keep four stages of the
// long operand in flight per CTA
template <int NT, bool LK>
__global__ void __launch_bounds__(SK_THREADS, 2) skinny_kernel(SkinnyArgs g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    skinny_body<NT, LK>(g, blockIdx.x, blockIdx.z, gridDim.z, smem_raw);
}

// Grouped launch: the row tiles (times K ranges) of many skinny products, tile_start[p]
// being the first CTA of problem p
template <int NT, bool LK>
__global__ void __launch_bounds__(SK_THREADS, 2)
    skinny_grouped_kernel(const SkinnyArgs* __restrict__ probs, const int* __restrict__ tile_start, int nprob) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ SkinnyArgs sg;
    __shared__ int sp;
    const int t = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile_start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        sp = lo;
        sg = probs[lo];
    }
    __syncthreads();
    const int local = t - tile_start[sp], rt = (sg.R + SK_TM - 1) / SK_TM;
    skinny_body<NT, LK>(sg, local % rt, local / rt, sg.nz, smem_raw);
}

__global__ void skinny_fold_kernel(SkinnyArgs g, int ks) {
    const int64_t rs = (int64_t)g.R * g.NS;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < rs; l += (int64_t)gridDim.x * blockDim.x) {
        double sum = 0.0;
        for (int z = 0; z < ks; z++) sum += g.ws[z * rs + l];
        const int r = (int)(l / g.NS), s = (int)(l % g.NS);
        const double v = g.alpha * sum;
        for (int a = 0; a < g.nvr; a++)
            for (int b = 0; b < g.nvs; b++) g.C[g.Cr[a][r] + g.Cs[b][s]] += g.vsign[a * g.nvs + b] * v;
    }
}

// ---------------------------------------------------------------------------
// Short products: M, N <= 64, long K.  Each warp of a CTA walks its own part of the CTA's
// K range, 16 k per step (8 for the widest shapes), loading the m8n8k4 fragments straight
// from global memory (a lane reads A[m = lane/4 + 8i][k] and B[k][n = lane/4 + 8j] for
// k = 4u + lane%4: 32-byte runs along k, or 64-byte runs along m / n, both whole
// sectors); the k offsets of the next step are fetched while the current step's data
// loads are in flight.  The eight warps' fragments are added in warp order in shared
// memory and the CTA writes one partial M x N product.
// ---------------------------------------------------------------------------
constexpr int SH_THREADS = 256;
constexpr int SH_KGRAN = 16 * (SH_THREADS / 32);   // kper is a multiple of this (128)

template <int MT, int NT>
__global__ void __launch_bounds__(SH_THREADS, MT * NT > 8 ? 1 : 2)
    short_grouped_kernel(const ShortDesc* __restrict__ descs, const int* __restrict__ cta_start, int nprob) {
    // steps of 16 k (8 for the widest shapes, whose loads of a step would not fit the registers)
    constexpr int SH_U = MT + NT <= 6 ? 4 : 2, SH_KSTEP = 4 * SH_U;
    __shared__ ShortDesc sd;
    __shared__ int sp;
    // the warps' fragments for the reduction (dynamic: 64 KB for 16 fragments)
    extern __shared__ __align__(16) unsigned char short_smem[];
    auto red = reinterpret_cast<double(*)[MT * 8 * NT * 8]>(short_smem);
    const int t = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cta_start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        sp = lo;
        sd = descs[lo];
    }
    __syncthreads();
    const ShortDesc& g = sd;
    const int local = t - cta_start[sp];
    const int fr = lane >> 2, fk = lane & 3;
    int64_t am[MT], bn[NT];
#pragma unroll
    for (int i = 0; i < MT; i++) am[i] = (8 * i + fr < g.M) ? __ldg(g.Am + 8 * i + fr) : -1;
#pragma unroll
    for (int j = 0; j < NT; j++) bn[j] = (8 * j + fr < g.N) ? __ldg(g.Bn + 8 * j + fr) : -1;

    const int kw = g.kper / (SH_THREADS / 32);               // k per warp (a multiple of 16)
    const int kb = local * g.kper + warp * kw;
    const int ke = min(g.K, kb + kw);
    double acc[MT][NT][2];
#pragma unroll
    for (int i = 0; i < MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    auto offsets = [&](int k0, int64_t* ak, int64_t* bk) {
#pragma unroll
        for (int u = 0; u < SH_U; u++) {
            const int k = k0 + 4 * u + fk;
            const bool ok = k < ke;
            ak[u] = !ok ? -1 : (g.ak_affine ? g.ak0 + g.ak_step * k : __ldg(g.Ak + k));
            bk[u] = !ok ? -1 : (g.bk_affine ? g.bk0 + g.bk_step * k : __ldg(g.Bk + k));
        }
    };
    int64_t ak[SH_U], bk[SH_U];
    if (kb < ke) offsets(kb, ak, bk);
    for (int k0 = kb; k0 < ke; k0 += SH_KSTEP) {
        double a[SH_U][MT], b[SH_U][NT];
#pragma unroll
        for (int u = 0; u < SH_U; u++) {
#pragma unroll
            for (int i = 0; i < MT; i++) a[u][i] = (ak[u] >= 0 && am[i] >= 0) ? __ldg(g.A + am[i] + ak[u]) : 0.0;
#pragma unroll
            for (int j = 0; j < NT; j++) b[u][j] = (bk[u] >= 0 && bn[j] >= 0) ? __ldg(g.B + bk[u] + bn[j]) : 0.0;
        }
        if (k0 + SH_KSTEP < ke) offsets(k0 + SH_KSTEP, ak, bk);
#pragma unroll
        for (int u = 0; u < SH_U; u++)
#pragma unroll
            for (int i = 0; i < MT; i++)
#pragma unroll
                for (int j = 0; j < NT; j++) dmma(acc[i][j][0], acc[i][j][1], a[u][i], b[u][j]);
    }
    // lane holds rows 8i + fr, columns 8j + 2 fk + {0, 1}
    constexpr int LDR = NT * 8;
#pragma unroll
    for (int i = 0; i < MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) red[warp][(8 * i + fr) * LDR + 8 * j + 2 * fk + h] = acc[i][j][h];
    __syncthreads();
    double* out = g.part + (int64_t)local * g.M * g.N;
    for (int e = tid; e < g.M * g.N; e += SH_THREADS) {
        const int m = e / g.N, n = e % g.N;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < SH_THREADS / 32; w++) s += red[w][m * LDR + n];
        out[e] = s;
    }
}

template <int MT, int NT>
void launch_short_t(const ShortDesc* d, const int* cta_start, int nprob, int total, cudaStream_t s) {
    constexpr int bytes = (SH_THREADS / 32) * MT * 8 * NT * 8 * (int)sizeof(double);
    set_smem_once((const void*)short_grouped_kernel<MT, NT>, bytes);
    short_grouped_kernel<MT, NT><<<total, SH_THREADS, bytes, s>>>(d, cta_start, nprob);
}

}  // namespace

// n-groups of 8 for a small extent (0: not a skinny product)
int skinny_groups(int M, int N) {
    const int small = std::min(M, N);
    if (small > 32) return 0;
    return small <= 8 ? 1 : (small <= 16 ? 2 : 4);
}

namespace {

// K-ranges for the skinny kernel: about two waves of CTAs, at least 16 k-chunks each
int skinny_ksplit(int R, int K, int nt) {
    (void)nt;
    const int tm = SK_TM, kc = SK_KC;
    const int64_t tiles = (R + tm - 1) / tm;
    if (tiles >= 2 * 148) return 1;
    const int64_t kchunks = (K + kc - 1) / kc;
    int64_t ks = (2 * 148 + tiles - 1) / tiles;
    ks = std::min<int64_t>(ks, kchunks / 16);
    ks = std::min<int64_t>(ks, 1024);
    return (int)std::max<int64_t>(ks, 1);
}

template <int NT, bool LK>
void launch_skinny_t(const SkinnyArgs& a, int ks, cudaStream_t s) {
    using Sh = SkinnyShape<NT, LK>;
    set_smem_once((const void*)skinny_kernel<NT, LK>, (int)Sh::bytes);
    dim3 grid((a.R + SK_TM - 1) / SK_TM, 1, ks);
    skinny_kernel<NT, LK><<<grid, SK_THREADS, Sh::bytes, s>>>(a);
}

template <int NT, bool LK>
void launch_skinny_grouped_t(const SkinnyArgs* d, const int* tile_start, int nprob, int tiles, cudaStream_t s) {
    using Sh = SkinnyShape<NT, LK>;
    set_smem_once((const void*)skinny_grouped_kernel<NT, LK>, (int)Sh::bytes);
    skinny_grouped_kernel<NT, LK><<<tiles, SK_THREADS, Sh::bytes, s>>>(d, tile_start, nprob);
}

void launch_skinny(const GemmArgs& g, int nt, cudaStream_t s) {
    bool lk;
    SkinnyArgs a = skinny_args(g, &lk);
    int ks = skinny_ksplit(a.R, a.K, nt);
    if (!g.ws || (int64_t)ks * a.R * a.NS > g.ws_elems) ks = 1;
    a.ws = g.ws;
    switch (nt * 2 + (lk ? 1 : 0)) {
        case 2: launch_skinny_t<1, false>(a, ks, s); break;
        case 3: launch_skinny_t<1, true>(a, ks, s); break;
        case 4: launch_skinny_t<2, false>(a, ks, s); break;
        case 5: launch_skinny_t<2, true>(a, ks, s); break;
        case 8: launch_skinny_t<4, false>(a, ks, s); break;
        default: launch_skinny_t<4, true>(a, ks, s); break;
    }
    COUNT_LAUNCH();
    if (ks > 1) {
        const int64_t rs = (int64_t)a.R * a.NS;
        const int nb = (int)std::min<int64_t>((rs + 255) / 256, 148 * 16);
        skinny_fold_kernel<<<nb, 256, 0, s>>>(a, ks);
        COUNT_LAUNCH();
    }
}

}  // namespace

SkinnyArgs skinny_args(const GemmArgs& g, bool* lk_out) {
    SkinnyArgs a;
    const bool long_a = g.M >= g.N;
    bool lk;
    a.C = g.C;
    a.alpha = g.alpha;
    a.K = g.K;
    if (long_a) {
        a.L = g.A; a.Lr = g.Am; a.Lk = g.Ak; a.S = g.B; a.Sk = g.Bk; a.Sn = g.Bn;
        a.R = g.M; a.NS = g.N; a.nvr = g.nvm; a.nvs = g.nvn;
        for (int v = 0; v < 2; v++) { a.Cr[v] = g.Cm[v]; a.Cs[v] = g.Cn[v]; }
        for (int i = 0; i < 4; i++) a.vsign[i] = g.vsign[i];
        lk = g.a_kcontig;
        a.lk_affine = g.ak_affine; a.lk0 = g.ak0; a.lk_step = g.ak_step;
        a.sk_affine = g.bk_affine; a.sk0 = g.bk0; a.sk_step = g.bk_step;
    } else {
        a.L = g.B; a.Lr = g.Bn; a.Lk = g.Bk; a.S = g.A; a.Sk = g.Ak; a.Sn = g.Am;
        a.R = g.N; a.NS = g.M; a.nvr = g.nvn; a.nvs = g.nvm;
        for (int v = 0; v < 2; v++) { a.Cr[v] = g.Cn[v]; a.Cs[v] = g.Cm[v]; }
        for (int r = 0; r < g.nvn; r++)
            for (int c = 0; c < g.nvm; c++) a.vsign[r * g.nvm + c] = g.vsign[c * g.nvn + r];
        lk = g.b_kcontig;
        a.lk_affine = g.bk_affine; a.lk0 = g.bk0; a.lk_step = g.bk_step;
        a.sk_affine = g.ak_affine; a.sk0 = g.ak0; a.sk_step = g.ak_step;
    }
    *lk_out = lk;
    return a;
}

int skinny_tiles(int R) { return (R + SK_TM - 1) / SK_TM; }

void skinny_grouped(const SkinnyArgs* d, const int* tile_start, int nprob, int tiles, int nt, bool lk, cudaStream_t s) {
    if (nprob <= 0 || tiles <= 0) return;
    switch (nt * 2 + (lk ? 1 : 0)) {
        case 2: launch_skinny_grouped_t<1, false>(d, tile_start, nprob, tiles, s); break;
        case 3: launch_skinny_grouped_t<1, true>(d, tile_start, nprob, tiles, s); break;
        case 4: launch_skinny_grouped_t<2, false>(d, tile_start, nprob, tiles, s); break;
        case 5: launch_skinny_grouped_t<2, true>(d, tile_start, nprob, tiles, s); break;
        case 8: launch_skinny_grouped_t<4, false>(d, tile_start, nprob, tiles, s); break;
        default: launch_skinny_grouped_t<4, true>(d, tile_start, nprob, tiles, s); break;
    }
    COUNT_LAUNCH();
}

namespace {

template <bool AK, bool BKc>
void launch_fp64(const GemmArgs& g, cudaStream_t s) {
    using S = Smem<AK, BKc>;
    set_smem_once((const void*)gemm_fp64_kernel<AK, BKc>, (int)S::bytes);
    int ks = fp64_ksplit(g.M, g.N, g.K, false);
    if (!g.ws || (int64_t)ks * g.M * g.N > g.ws_elems) ks = 1;
    if ((g.M + BM - 1) / BM > 65535) throw std::runtime_error("FP64 GEMM: M too large for the grid");
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, ks);
    gemm_fp64_kernel<AK, BKc><<<grid, THREADS, S::bytes, s>>>(g);
    COUNT_LAUNCH();
    if (ks > 1) {
        const int64_t mn = (int64_t)g.M * g.N;
        int nb = (int)std::min<int64_t>((mn + 255) / 256, 148 * 16);
        splitk_fold_kernel<<<nb, 256, 0, s>>>(g, ks);
        COUNT_LAUNCH();
    }
}

}  // namespace

// Few output tiles and a long K: split K so that about two waves of CTAs stream the
// operands; every split keeps at least 512 k.
int fp64_ksplit(int M, int N, int K, bool skinny_ok) {
    if (const int nt = skinny_ok ? skinny_groups(M, N) : 0) return skinny_ksplit(std::max(M, N), K, nt);
    const int64_t tiles = (int64_t)((M + BM - 1) / BM) * ((N + BN - 1) / BN);
    const int ktiles = (K + BK - 1) / BK;
    if (tiles >= 148) return 1;
    int64_t ks = (2 * 148 + tiles - 1) / tiles;
    ks = std::min<int64_t>(ks, ktiles / 32);
    ks = std::min<int64_t>(ks, 256);
    return (int)std::max<int64_t>(ks, 1);
}

void gemm_fp64(const GemmArgs& g, cudaStream_t s) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0) return;
    if (const int nt = g.skinny_ok ? skinny_groups(g.M, g.N) : 0) {
        launch_skinny(g, nt, s);
        return;
    }
    if (g.a_kcontig) {
        if (g.b_kcontig) launch_fp64<true, true>(g, s);
        else launch_fp64<true, false>(g, s);
    } else {
        if (g.b_kcontig) launch_fp64<false, true>(g, s);
        else launch_fp64<false, false>(g, s);
    }
}

int fp64_tiles(int M, int N) { return ((M + BM - 1) / BM) * ((N + BN - 1) / BN); }

void splitk_fold(const GemmArgs& g, int ks, cudaStream_t s) {
    const int64_t mn = (int64_t)g.M * g.N;
    if (mn <= 0 || ks <= 1) return;
    const int nb = (int)std::min<int64_t>((mn + 255) / 256, 148 * 16);
    splitk_fold_kernel<<<nb, 256, 0, s>>>(g, ks);
    COUNT_LAUNCH();
}

namespace {
template <bool AK, bool BKc>
void launch_grouped_t(const GemmArgs* probs, const int* tile_start, int nprob, int total_tiles, cudaStream_t s) {
    using S = Smem<AK, BKc>;
    set_smem_once((const void*)gemm_fp64_grouped_kernel<AK, BKc>, (int)S::bytes);
    gemm_fp64_grouped_kernel<AK, BKc><<<total_tiles, THREADS, S::bytes, s>>>(probs, tile_start, nprob);
}
}  // namespace

void gemm_fp64_grouped(const GemmArgs* probs, const int* tile_start, int nprob, int total_tiles, bool a_kcontig,
                       bool b_kcontig, cudaStream_t s) {
    if (nprob <= 0 || total_tiles <= 0) return;
    if (a_kcontig) {
        if (b_kcontig) launch_grouped_t<true, true>(probs, tile_start, nprob, total_tiles, s);
        else launch_grouped_t<true, false>(probs, tile_start, nprob, total_tiles, s);
    } else {
        if (b_kcontig) launch_grouped_t<false, true>(probs, tile_start, nprob, total_tiles, s);
        else launch_grouped_t<false, false>(probs, tile_start, nprob, total_tiles, s);
    }
    COUNT_LAUNCH();
}

std::pair<int, int> short_shape(int M, int N) {
    if (M <= 0 || N <= 0 || M > 64 || N > 64) return {0, 0};
    auto frag = [](int x) { return x <= 8 ? 1 : (x <= 16 ? 2 : (x <= 32 ? 4 : 8)); };
    const int mt = frag(M), nt = frag(N);
    if (mt * nt > 16) return {0, 0};
    return {mt, nt};
}

int short_ctas(int K, int* kper) {
    // about 2048 k per CTA (eight warps, 16 steps of 16 k each), at most 512 CTAs
    int ctas = std::max(1, std::min(512, (K + 2047) / 2048));
    int per = (K + ctas - 1) / ctas;
    per = (per + SH_KGRAN - 1) / SH_KGRAN * SH_KGRAN;
    ctas = (K + per - 1) / per;
    *kper = per;
    return ctas;
}

void short_grouped(const ShortDesc* d, const int* cta_start, int nprob, int total_ctas, int mt, int nt,
                   cudaStream_t s) {
    if (nprob <= 0 || total_ctas <= 0) return;
    switch (mt * 16 + nt) {
        case 0x11: launch_short_t<1, 1>(d, cta_start, nprob, total_ctas, s); break;
        case 0x12: launch_short_t<1, 2>(d, cta_start, nprob, total_ctas, s); break;
        case 0x14: launch_short_t<1, 4>(d, cta_start, nprob, total_ctas, s); break;
        case 0x18: launch_short_t<1, 8>(d, cta_start, nprob, total_ctas, s); break;
        case 0x21: launch_short_t<2, 1>(d, cta_start, nprob, total_ctas, s); break;
        case 0x22: launch_short_t<2, 2>(d, cta_start, nprob, total_ctas, s); break;
        case 0x24: launch_short_t<2, 4>(d, cta_start, nprob, total_ctas, s); break;
        case 0x41: launch_short_t<4, 1>(d, cta_start, nprob, total_ctas, s); break;
        case 0x42: launch_short_t<4, 2>(d, cta_start, nprob, total_ctas, s); break;
        case 0x81: launch_short_t<8, 1>(d, cta_start, nprob, total_ctas, s); break;
        case 0x28: launch_short_t<2, 8>(d, cta_start, nprob, total_ctas, s); break;
        case 0x44: launch_short_t<4, 4>(d, cta_start, nprob, total_ctas, s); break;
        case 0x82: launch_short_t<8, 2>(d, cta_start, nprob, total_ctas, s); break;
        default: throw std::runtime_error("short product: unsupported fragment shape");
    }
    COUNT_LAUNCH();
}

void fold_groups(const FoldDesc* d, const int* group_start, int ngroups, cudaStream_t s) {
    if (ngroups <= 0) return;
    fold_groups_kernel<<<ngroups, 256, 0, s>>>(d, group_start);
    COUNT_LAUNCH();
}

// ---------------------------------------------------------------------------
// elementwise and reductions
// ---------------------------------------------------------------------------
namespace {

constexpr int EW_THREADS = 256;

inline int ew_blocks(int64_t n) {
    int64_t b = (n + EW_THREADS - 1) / EW_THREADS;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

__global__ void sum_strided_kernel(const double* __restrict__ A, double* __restrict__ C, StridedArgs a,
                                   double alpha) {
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < a.total;
         l += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = l, oa = 0, oc = 0;
        for (int d = 0; d < a.ndim; d++) {
            int64_t x = r % a.len[d];
            r /= a.len[d];
            oa += x * a.sA[d];
            oc += x * a.sB[d];
        }
        C[oc] += alpha * A[oa];
    }
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    v = 0;
    if (threadIdx.x < (blockDim.x >> 5)) v = red[threadIdx.x];
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_max(double v) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    v = 0;
    if (threadIdx.x < (blockDim.x >> 5)) v = red[threadIdx.x];
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// deterministic two-pass reductions: blocks write partials, one block folds them
__global__ void dot_strided_kernel(const double* __restrict__ A, const double* __restrict__ B, StridedArgs a,
                                   double* partial) {
    double s = 0;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < a.total;
         l += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = l, oa = 0, ob = 0;
        for (int d = 0; d < a.ndim; d++) {
            int64_t x = r % a.len[d];
            r /= a.len[d];
            oa += x * a.sA[d];
            ob += x * a.sB[d];
        }
        s += A[oa] * B[ob];
    }
    s = block_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void fold_sum_kernel(const double* partial, int n, double alpha, double* out) {
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
    s = block_sum(s);
    if (threadIdx.x == 0) out[0] += alpha * s;
}

__global__ void norm_kernel(const double* __restrict__ X, int64_t n, int p, double* partial) {
    double s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = X[i];
        if (p == 0) s = fmax(s, fabs(x));
        else if (p == 1) s += fabs(x);
        else s += x * x;
    }
    s = p == 0 ? block_max(s) : block_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void fold_norm_kernel(const double* partial, int n, int p, double w, double* out) {
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = p == 0 ? fmax(s, partial[i]) : s + partial[i];
    s = p == 0 ? block_max(s) : block_sum(s);
    if (threadIdx.x == 0) out[0] = p == 0 ? fmax(out[0], s) : out[0] + w * s;
}

__global__ void scale_kernel(double* X, int64_t n, double beta) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        X[i] = beta == 0.0 ? 0.0 : beta * X[i];
}

__global__ void fill_kernel(double* X, int64_t n, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        X[i] = v;
}

__global__ void axpby_kernel(const double* __restrict__ x, double* __restrict__ y, int64_t n, double a, double b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
}

__device__ __forceinline__ double den_of(const WeightArgs& w, int64_t l) {
    double den = 0;
    int64_t r = l;
    for (int d = 0; d < w.ndim; d++) {
        int64_t x = r % w.len[d];
        r /= w.len[d];
        den += w.d[d][x];
    }
    return den;
}

__global__ void weight_kernel(double* X, WeightArgs w, double shift) {
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < w.total;
         l += (int64_t)gridDim.x * blockDim.x) {
        double den = den_of(w, l) + shift;
        X[l] = fabs(den) < 1e-4 ? 0.0 : X[l] / den;
    }
}

// z = z/den (0 if |den| < 1e-4), t += z, block max |z|
__global__ void update_kernel(double* __restrict__ Z, double* __restrict__ T, WeightArgs w, double* partial) {
    double mx = 0;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < w.total;
         l += (int64_t)gridDim.x * blockDim.x) {
        double den = den_of(w, l);
        double z = fabs(den) < 1e-4 ? 0.0 : Z[l] / den;
        Z[l] = z;
        T[l] += z;
        mx = fmax(mx, fabs(z));
    }
    mx = block_max(mx);
    if (threadIdx.x == 0) partial[blockIdx.x] = mx;
}

__global__ void kv_write_kernel(double* X, const int64_t* keys, const double* vals, int64_t n, double a, double b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double* p = X + keys[i];
        *p = (b == 0.0 ? 0.0 : b * *p) + a * vals[i];
    }
}

__global__ void kv_read_kernel(const double* X, const int64_t* keys, double* vals, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        vals[i] = X[keys[i]];
}

// batched dot: partial[b * ny + j] = sum over the block's range of x * ys[j]
__global__ void dot_batch_kernel(const double* __restrict__ x, const double* const* ys, int ny, int64_t n,
                                 double* partial) {
    double s[16];
    for (int j = 0; j < 16; j++) s[j] = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double xv = x[i];
        for (int j = 0; j < ny; j++) s[j] += xv * ys[j][i];
    }
    for (int j = 0; j < ny; j++) {
        double t = block_sum(s[j]);
        if (threadIdx.x == 0) partial[blockIdx.x * ny + j] = t;
    }
}

__global__ void fold_batch_kernel(const double* partial, int nb, int ny, double w, double* out) {
    for (int j = 0; j < ny; j++) {
        double s = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[b * ny + j];
        s = block_sum(s);
        if (threadIdx.x == 0) out[j] += w * s;
    }
}

__global__ void lincomb_kernel(double* __restrict__ out1, int64_t n1, double* __restrict__ out2, int64_t n2,
                               const double* const* xs, const double* c, int nx) {
    const int64_t n = n1 + n2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int j = 0; j < nx; j++) {
            double cj = c[j];
            if (cj != 0.0) s += cj * xs[j][i];
        }
        if (i < n1) out1[i] = s;
        else out2[i - n1] = s;
    }
}

// Scratch for the two-pass reductions, one buffer per stream: work on one stream is
// ordered, and each fold consumes its partials before the next reduction on that
// stream overwrites them.  Buffers live until process exit.
}  // namespace

namespace {
std::mutex g_partial_mu;
std::map<std::pair<int, cudaStream_t>, double*> g_partial;
}  // namespace

double* partial_buffer(cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_partial_mu);
    auto key = std::make_pair(dev, s);
    auto it = g_partial.find(key);
    if (it != g_partial.end()) return it->second;
    double* p = nullptr;
    cudaMalloc(&p, sizeof(double) * 148 * 16 * 16);
    g_partial[key] = p;
    return p;
}

namespace {

__device__ __forceinline__ int find_problem(const int64_t* __restrict__ cs, int n, int64_t c) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cs[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) sum_batched_kernel(const SumDesc* __restrict__ d, const int64_t* __restrict__ cs,
                                                          int n) {
    __shared__ int sp;
    __shared__ double tile[32][33];
    const int64_t c = blockIdx.x;
    if (threadIdx.x == 0) sp = find_problem(cs, n, c);
    __syncthreads();
    const SumDesc& D = d[sp];
    if (D.tiled) {
        // two 32 x 32 tiles over (p0, pc): read along p0 (A-contiguous), write along pc
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
        const int64_t l0 = D.len[D.p0], lc = D.len[D.pc];
        const int64_t t0n = (l0 + 31) / 32, tcn = (lc + 31) / 32;
        for (int tt = 0; tt < 2; tt++) {
            const int64_t t = (c - cs[sp]) * 2 + tt;
            if (t >= D.ntiles) break;   // uniform across the CTA
            int64_t r = t;
            const int64_t t0 = r % t0n;
            r /= t0n;
            const int64_t tc = r % tcn;
            r /= tcn;
            int64_t oa = 0, oc = 0;
            for (int k = 0; k < D.ndim; k++) {
                if (k == D.p0 || k == D.pc) continue;
                const int64_t x = r % D.len[k];
                r /= D.len[k];
                oa += x * D.sA[k];
                oc += x * D.sC[k];
            }
            const int64_t x0 = t0 * 32 + tx;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int64_t xc = tc * 32 + ty + 8 * q;
                tile[ty + 8 * q][tx] = (x0 < l0 && xc < lc) ? D.A[oa + x0 * D.sA[D.p0] + xc * D.sA[D.pc]] : 0.0;
            }
            __syncthreads();
            const int64_t xc = tc * 32 + tx;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int64_t y0 = t0 * 32 + ty + 8 * q;
                if (y0 < l0 && xc < lc) D.C[oc + y0 * D.sC[D.p0] + xc * D.sC[D.pc]] += D.alpha * tile[tx][ty + 8 * q];
            }
            __syncthreads();
        }
        return;
    }
    // a thread's elements in batches of four: the offsets, then the loads, then the stores,
    // so that the loads of a batch are in flight together (batches of four keep the
    // registers, and with them the occupancy of the tiled path of this kernel, low)
    constexpr int PER = 4;
    for (int half = 0; half < kBatchChunk / (256 * PER); half++) {
    const int64_t base = (c - cs[sp]) * kBatchChunk + half * 256 * PER;
    int64_t oa[PER], oc[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int64_t l = base + threadIdx.x + q * 256;
        oa[q] = -1;
        oc[q] = 0;
        if (l >= D.total) continue;
        int64_t a = 0, cc = 0;
        if (D.fast) {
            uint32_t r = (uint32_t)l;
            for (int k = 0; k < D.ndim; k++) {
                const uint32_t qq = (uint32_t)(((uint64_t)__umulhi(r, D.dmul[k]) + r) >> D.dshr[k]);
                const uint32_t x = r - qq * (uint32_t)D.len[k];
                a += (int64_t)x * D.sA[k];
                cc += (int64_t)x * D.sC[k];
                r = qq;
            }
        } else {
            int64_t r = l;
            for (int k = 0; k < D.ndim; k++) {
                const int64_t x = r % D.len[k];
                r /= D.len[k];
                a += x * D.sA[k];
                cc += x * D.sC[k];
            }
        }
        oa[q] = a;
        oc[q] = cc;
    }
    double va[PER], vc[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        va[q] = oa[q] >= 0 ? D.A[oa[q]] : 0.0;
        vc[q] = oa[q] >= 0 ? D.C[oc[q]] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < PER; q++)
        if (oa[q] >= 0) D.C[oc[q]] = vc[q] + D.alpha * va[q];
    }
}

__global__ void __launch_bounds__(256) scale_batched_kernel(const ScaleDesc* __restrict__ d,
                                                            const int64_t* __restrict__ cs, int n) {
    __shared__ int sp;
    const int64_t c = blockIdx.x;
    if (threadIdx.x == 0) sp = find_problem(cs, n, c);
    __syncthreads();
    const ScaleDesc& D = d[sp];
    const int64_t base = (c - cs[sp]) * kBatchChunk;
    for (int i = threadIdx.x; i < kBatchChunk; i += blockDim.x) {
        const int64_t l = base + i;
        if (l >= D.n) break;
        D.X[l] = D.beta == 0.0 ? 0.0 : D.beta * D.X[l];
    }
}

// Tau of one chunk of one block (tau_kernel's arithmetic)
__global__ void __launch_bounds__(256) tau_batched_kernel(const TauArgs* __restrict__ d, const int64_t* __restrict__ cs,
                                                          int n) {
    __shared__ int sp;
    const int64_t c = blockIdx.x;
    if (threadIdx.x == 0) sp = find_problem(cs, n, c);
    __syncthreads();
    const TauArgs& a = d[sp];
    const int64_t la = a.len[0], lb = a.len[1], li = a.len[2], lj = a.len[3];
    const int64_t total = la * lb * li * lj;
    const int64_t base = (c - cs[sp]) * kBatchChunk;
    for (int i = threadIdx.x; i < kBatchChunk; i += blockDim.x) {
        const int64_t l = base + i;
        if (l >= total) break;
        int64_t r = l;
        const int64_t x = r % la;
        r /= la;
        const int64_t y = r % lb;
        r /= lb;
        const int64_t ii = r % li;
        const int64_t j = r / li;
        double v = a.t2[l];
        if (a.t1ai) v += a.t1ai[x + la * ii] * a.t1bj[y + lb * j];
        if (a.t1aj) v -= a.t1aj[x + la * j] * a.t1bi[y + lb * ii];
        a.tau[l] = v;
    }
}

// Jacobi update of one chunk of one block; the residual max goes to red_max through an
// atomic max on the bits of non-negative doubles (order-independent)
__global__ void __launch_bounds__(256) update_batched_kernel(const UpdateDesc* __restrict__ d,
                                                             const int64_t* __restrict__ cs, int n, double* red_max) {
    __shared__ int sp;
    const int64_t c = blockIdx.x;
    if (threadIdx.x == 0) sp = find_problem(cs, n, c);
    __syncthreads();
    const UpdateDesc& D = d[sp];
    const int64_t base = (c - cs[sp]) * kBatchChunk;
    double mx = 0;
    for (int i = threadIdx.x; i < kBatchChunk; i += blockDim.x) {
        const int64_t l = base + i;
        if (l >= D.w.total) break;
        const double den = den_of(D.w, l);
        const double z = fabs(den) < 1e-4 ? 0.0 : D.Z[l] / den;
        D.Z[l] = z;
        D.T[l] += z;
        mx = fmax(mx, fabs(z));
    }
    mx = block_max(mx);
    if (threadIdx.x == 0 && mx > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(red_max), (unsigned long long)__double_as_longlong(mx));
}

// dot of one chunk of one block into part[c]
__global__ void __launch_bounds__(256) dot_batched_kernel(const DotDesc* __restrict__ d, const int64_t* __restrict__ cs,
                                                          int n, double* part) {
    __shared__ int sp;
    const int64_t c = blockIdx.x;
    if (threadIdx.x == 0) sp = find_problem(cs, n, c);
    __syncthreads();
    const DotDesc& D = d[sp];
    const int64_t base = (c - cs[sp]) * kBatchChunk;
    double acc = 0;
    // batches of four elements: the offsets first, then the loads (in flight together)
    constexpr int PER = 4;
    for (int half = 0; half < kBatchChunk / (256 * PER); half++) {
    int64_t oa[PER], ob[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int64_t l = base + half * 256 * PER + threadIdx.x + q * 256;
        oa[q] = -1;
        ob[q] = 0;
        if (l >= D.total) continue;
        int64_t a = 0, b = 0;
        if (D.fast) {
            uint32_t r = (uint32_t)l;
            for (int k = 0; k < D.ndim; k++) {
                const uint32_t qq = (uint32_t)(((uint64_t)__umulhi(r, D.dmul[k]) + r) >> D.dshr[k]);
                const uint32_t x = r - qq * (uint32_t)D.len[k];
                a += (int64_t)x * D.sA[k];
                b += (int64_t)x * D.sB[k];
                r = qq;
            }
        } else {
            int64_t r = l;
            for (int k = 0; k < D.ndim; k++) {
                const int64_t x = r % D.len[k];
                r /= D.len[k];
                a += x * D.sA[k];
                b += x * D.sB[k];
            }
        }
        oa[q] = a;
        ob[q] = b;
    }
#pragma unroll
    for (int q = 0; q < PER; q++)
        if (oa[q] >= 0) acc += D.A[oa[q]] * D.B[ob[q]];
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[c] = D.alpha * acc;
}

}  // namespace

// multiply-shift division by every extent (Granlund-Montgomery, round-up variant): for
// 1 <= len < 2^31, shr = ceil(log2 len), mul = floor(2^32 (2^shr - len) / len) + 1 gives
// x / len = (umulhi(x, mul) + x) >> shr for every x < 2^32
void plan_divisors(const int64_t* lens, int ndim, int64_t total, int& fast, uint32_t* dmul, uint32_t* dshr) {
    fast = total < ((int64_t)1 << 31) ? 1 : 0;
    for (int k = 0; k < ndim && fast; k++) {
        const uint64_t len = (uint64_t)lens[k];
        if (len < 1 || len >= ((uint64_t)1 << 31)) {
            fast = 0;
            break;
        }
        uint32_t l = 0;
        while (((uint64_t)1 << l) < len) l++;
        dshr[k] = l;
        dmul[k] = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << l) - len)) / len + 1);
    }
}

void sum_plan_tiles(SumDesc& d) {
    d.tiled = 0;
    plan_divisors(d.len, d.ndim, d.total, d.fast, d.dmul, d.dshr);
    if (d.ndim < 2) return;
    int p0 = 0, pc = 0;
    for (int k = 1; k < d.ndim; k++) {
        if (d.sA[k] < d.sA[p0]) p0 = k;
        if (d.sC[k] < d.sC[pc]) pc = k;
    }
    if (p0 == pc || d.len[p0] < 8 || d.len[pc] < 8) return;
    d.tiled = 1;
    d.p0 = p0;
    d.pc = pc;
    d.ntiles = ((d.len[p0] + 31) / 32) * ((d.len[pc] + 31) / 32);
    for (int k = 0; k < d.ndim; k++)
        if (k != p0 && k != pc) d.ntiles *= d.len[k];
}

void sum_batched(const SumDesc* d, const int64_t* chunk_start, int n, int64_t chunks, cudaStream_t s) {
    if (n <= 0 || chunks <= 0) return;
    sum_batched_kernel<<<(unsigned)chunks, 256, 0, s>>>(d, chunk_start, n);
    COUNT_LAUNCH();
}

void tau_batched(const TauArgs* d, const int64_t* chunk_start, int n, int64_t chunks, cudaStream_t s) {
    if (n <= 0 || chunks <= 0) return;
    tau_batched_kernel<<<(unsigned)chunks, 256, 0, s>>>(d, chunk_start, n);
    COUNT_LAUNCH();
}

void update_batched(const UpdateDesc* d, const int64_t* chunk_start, int n, int64_t chunks, double* red_max,
                    cudaStream_t s) {
    if (n <= 0 || chunks <= 0) return;
    update_batched_kernel<<<(unsigned)chunks, 256, 0, s>>>(d, chunk_start, n, red_max);
    COUNT_LAUNCH();
}

void dot_batched(const DotDesc* d, const int64_t* chunk_start, int n, int64_t chunks, double* part, double* out,
                 cudaStream_t s) {
    if (n <= 0 || chunks <= 0) return;
    dot_batched_kernel<<<(unsigned)chunks, 256, 0, s>>>(d, chunk_start, n, part);
    fold_sum_kernel<<<1, 1024, 0, s>>>(part, (int)chunks, 1.0, out);
    COUNT_LAUNCH();
    COUNT_LAUNCH();
}

void scale_batched(const ScaleDesc* d, const int64_t* chunk_start, int n, int64_t chunks, cudaStream_t s) {
    if (n <= 0 || chunks <= 0) return;
    scale_batched_kernel<<<(unsigned)chunks, 256, 0, s>>>(d, chunk_start, n);
    COUNT_LAUNCH();
}

void release_stream_buffers(cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_partial_mu);
    auto it = g_partial.find(std::make_pair(dev, s));
    if (it == g_partial.end()) return;
    cudaStreamSynchronize(s);
    cudaFree(it->second);
    g_partial.erase(it);
}

void sum_strided(const double* A, double* C, const StridedArgs& a, double alpha, cudaStream_t s) {
    if (a.total <= 0) return;
    sum_strided_kernel<<<ew_blocks(a.total), EW_THREADS, 0, s>>>(A, C, a, alpha);
    COUNT_LAUNCH();
}

void dot_strided(const double* A, const double* B, const StridedArgs& a, double alpha, double* out,
                 cudaStream_t s) {
    if (a.total <= 0) return;
    int nb = ew_blocks(a.total);
    double* part = partial_buffer(s);
    dot_strided_kernel<<<nb, EW_THREADS, 0, s>>>(A, B, a, part);
    fold_sum_kernel<<<1, 1024, 0, s>>>(part, nb, alpha, out);
    COUNT_LAUNCH();
    COUNT_LAUNCH();
}

void scale(double* X, int64_t n, double beta, cudaStream_t s) {
    if (n <= 0 || beta == 1.0) return;
    scale_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(X, n, beta);
    COUNT_LAUNCH();
}

void fill(double* X, int64_t n, double val, cudaStream_t s) {
    if (n <= 0) return;
    fill_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(X, n, val);
    COUNT_LAUNCH();
}

void norm_accum(const double* X, int64_t n, int p, double w, double* out, cudaStream_t s) {
    if (n <= 0) return;
    int nb = ew_blocks(n);
    double* part = partial_buffer(s);
    norm_kernel<<<nb, EW_THREADS, 0, s>>>(X, n, p, part);
    fold_norm_kernel<<<1, 1024, 0, s>>>(part, nb, p, w, out);
    COUNT_LAUNCH();
    COUNT_LAUNCH();
}

void axpby(const double* x, double* out, int64_t n, double alpha, double beta, cudaStream_t s) {
    if (n <= 0) return;
    axpby_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(x, out, n, alpha, beta);
    COUNT_LAUNCH();
}

void weight_block(double* X, const WeightArgs& w, double shift, cudaStream_t s) {
    if (w.total <= 0) return;
    weight_kernel<<<ew_blocks(w.total), EW_THREADS, 0, s>>>(X, w, shift);
    COUNT_LAUNCH();
}

void update_block(double* Z, double* T, const WeightArgs& w, double* red_max, cudaStream_t s) {
    if (w.total <= 0) return;
    int nb = ew_blocks(w.total);
    double* part = partial_buffer(s);
    update_kernel<<<nb, EW_THREADS, 0, s>>>(Z, T, w, part);
    fold_norm_kernel<<<1, 1024, 0, s>>>(part, nb, 0, 1.0, red_max);
    COUNT_LAUNCH();
    COUNT_LAUNCH();
}

void kv_write(double* X, const int64_t* keys, const double* vals, int64_t n, double alpha, double beta,
              cudaStream_t s) {
    if (n <= 0) return;
    kv_write_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(X, keys, vals, n, alpha, beta);
    COUNT_LAUNCH();
}

void kv_read(const double* X, const int64_t* keys, double* vals, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    kv_read_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(X, keys, vals, n);
    COUNT_LAUNCH();
}

void dot_batch(const double* x, const double* const* ys, int ny, int64_t n, double w, double* out,
               cudaStream_t s) {
    if (n <= 0 || ny <= 0) return;
    int nb = ew_blocks(n);
    double* part = partial_buffer(s);
    dot_batch_kernel<<<nb, EW_THREADS, 0, s>>>(x, ys, ny, n, part);
    fold_batch_kernel<<<1, 1024, 0, s>>>(part, nb, ny, w, out);
    COUNT_LAUNCH();
    COUNT_LAUNCH();
}

void lincomb(double* out1, int64_t n1, double* out2, int64_t n2, const double* const* xs, const double* c, int nx,
             cudaStream_t s) {
    if (n1 + n2 <= 0) return;
    lincomb_kernel<<<ew_blocks(n1 + n2), EW_THREADS, 0, s>>>(out1, n1, out2, n2, xs, c, nx);
    COUNT_LAUNCH();
}


// ---------------------------------------------------------------------------
// device-resident DIIS
// ---------------------------------------------------------------------------
namespace {

__global__ void diis_advance_kernel(int* st, int order) {
    st[0] = (st[0] + 1) % order;
    st[1] = min(st[1] + 1, order);
}

__global__ void diis_store_kernel(const int* st, const double* const* xs, const double* const* dxs,
                                  const double* __restrict__ t1, int64_t n1, const double* __restrict__ t2, int64_t n2,
                                  const double* __restrict__ z1, const double* __restrict__ z2) {
    const int h = st[0];
    double* x = const_cast<double*>(xs[h]);
    double* dx = const_cast<double*>(dxs[h]);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n1 + n2; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n1) {
            x[i] = t1[i];
            dx[i] = z1[i];
        } else {
            x[i] = t2[i - n1];
            dx[i] = z2[i - n1];
        }
    }
}

__global__ void diis_dots_kernel(const int* st, const double* const* dxs, int order, int64_t off, int64_t len,
                                 double* partial) {
    const double* x = dxs[st[0]] + off;
    double s[16];
    for (int j = 0; j < 16; j++) s[j] = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
        double xv = x[i];
#pragma unroll
        for (int j = 0; j < 16; j++)
            if (j < order) s[j] += xv * dxs[j][off + i];
    }
    for (int j = 0; j < order; j++) {
        double t = block_sum(s[j]);
        if (threadIdx.x == 0) partial[blockIdx.x * order + j] = t;
    }
}

// Gaussian elimination with partial pivoting on an m x m system (m <= 17); false if a
// pivot is exactly zero
__device__ bool small_solve(double (*A)[17], double* b, int m) {
    for (int k = 0; k < m; k++) {
        int p = k;
        for (int i = k + 1; i < m; i++)
            if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
        if (A[p][k] == 0.0) return false;
        if (p != k) {
            for (int j = 0; j < m; j++) {
                double t = A[k][j];
                A[k][j] = A[p][j];
                A[p][j] = t;
            }
            double t = b[k];
            b[k] = b[p];
            b[p] = t;
        }
        for (int i = k + 1; i < m; i++) {
            double f = A[i][k] / A[k][k];
            for (int j = k; j < m; j++) A[i][j] -= f * A[k][j];
            b[i] -= f * b[k];
        }
    }
    for (int k = m - 1; k >= 0; k--) {
        double t = b[k];
        for (int j = k + 1; j < m; j++) t -= A[k][j] * b[j];
        b[k] = t / A[k][k];
    }
    return true;
}

__global__ void diis_solve_kernel(int* st, double* e, double* c, const double* dots, int order) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int ld = order + 1;
    const int head = st[0], cnt = st[1];
    for (int j = 0; j < order; j++) {
        e[head * ld + j] = dots[j];
        e[j * ld + head] = dots[j];
    }
    for (int j = 0; j <= order; j++) c[j] = 0.0;
    // diis.hpp:151: a single vector gives no extrapolation
    if (cnt == 1) {
        c[head] = 1.0;
        return;
    }
    // diis.hpp:153: --start > 1 delays the extrapolation
    int start = --st[2];
    if (start > 1) {
        c[head] = 1.0;
        return;
    }
    double A[17][17], b[17];
    auto slot = [&](int age) { return ((head - age) % order + order) % order; };
    auto fill = [&](double shift) {
        for (int i = 0; i < cnt; i++) {
            for (int j = 0; j < cnt; j++) A[i][j] = e[slot(i) * ld + slot(j)];
            A[i][i] += shift;
            A[i][cnt] = -1.0;
            A[cnt][i] = -1.0;
            b[i] = 0.0;
        }
        A[cnt][cnt] = 0.0;
        b[cnt] = -1.0;
    };
    fill(0.0);
    bool ok = small_solve(A, b, cnt + 1);
    if (!ok) {
        // diis.hpp:177-185: shift the diagonal by eps * e[n-1][n-1] and retry
        double eps = e[slot(cnt - 1) * ld + slot(cnt - 1)] * 2.220446049250313e-16;
        fill(eps);
        ok = small_solve(A, b, cnt + 1);
    }
    if (!ok) {
        st[3] = 1;
        c[head] = 1.0;
        return;
    }
    for (int i = 0; i < cnt; i++) c[slot(i)] = b[i];
}

// one piece of a caller's (x, dx) pair into the head slot at offset `off`
__global__ void diis_store_segment_kernel(const int* st, const double* const* xs, const double* const* dxs,
                                          int64_t off, const double* __restrict__ x, const double* __restrict__ dx,
                                          int64_t len) {
    const int h = st[0];
    double* rx = const_cast<double*>(xs[h]) + off;
    double* rdx = const_cast<double*>(dxs[h]) + off;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
        rx[i] = x[i];
        rdx[i] = dx[i];
    }
}

// out[i] = sum_j c[j] * xs[j][off + i]
__global__ void lincomb_segment_kernel(double* __restrict__ out, int64_t len, const double* const* xs, int64_t off,
                                       const double* c, int nx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int j = 0; j < nx; j++) {
            double cj = c[j];
            if (cj != 0.0) s += cj * xs[j][off + i];
        }
        out[i] = s;
    }
}

// diis.hpp:155-161: while the start counter is above 1 (and two vectors are stored), the
// stored newest x becomes (damping - 1) x_0 + damping x_1
__global__ void diis_damp_kernel(const int* st, const double* const* xs, int order, int64_t len, double damping) {
    if (st[1] < 2 || st[2] <= 1) return;
    const int h = st[0], p = (st[0] - 1 + order) % order;
    double* x0 = const_cast<double*>(xs[h]);
    const double* x1 = xs[p];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
        x0[i] = (damping - 1.0) * x0[i] + damping * x1[i];
}

}  // namespace

namespace {

__device__ __forceinline__ void tri_decode(int64_t p, int64_t& x, int64_t& y) {
    // p = y(y-1)/2 + x with 0 <= x < y
    int64_t yy = (int64_t)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while (yy * (yy - 1) / 2 > p) yy--;
    while ((yy + 1) * yy / 2 <= p) yy++;
    y = yy;
    x = p - yy * (yy - 1) / 2;
}

__global__ void pack_vvvv_kernel(double* V, int kab, int kcd, int n0, int n1, int n2, int n3, int64_t scd,
                                 const double* __restrict__ tJ, const double* __restrict__ tK, int a0, int a1,
                                 bool J, bool K) {
    const int ca = a1 - a0;
    const int64_t ncd = kcd == 1 ? (int64_t)n2 * (n2 - 1) / 2 : (int64_t)n2 * n3;
    const int64_t total = (int64_t)ca * n1 * ncd;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < total; l += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = l;
        int a = (int)(r % ca) + a0;
        r /= ca;
        int b = (int)(r % n1);
        int64_t pcd = r / n1;
        if (kab == 1 && b <= a) continue;
        int64_t c, d;
        if (kcd == 1) tri_decode(pcd, c, d);
        else {
            c = pcd % n2;
            d = pcd / n2;
        }
        int64_t pab = kab == 1 ? (int64_t)b * (b - 1) / 2 + a : (int64_t)a + (int64_t)n0 * b;
        const int64_t ap = a - a0;
        double v = 0;
        if (J) v += tJ[ap + ca * (c + (int64_t)n2 * (b + (int64_t)n1 * d))];
        if (K) v -= tK[ap + ca * (d + (int64_t)n3 * (b + (int64_t)n1 * c))];
        V[pab + scd * pcd] = v;
    }
}

}  // namespace

namespace {
__global__ void tau_kernel(TauArgs a) {
    const int64_t la = a.len[0], lb = a.len[1], li = a.len[2], lj = a.len[3];
    const int64_t n = la * lb * li * lj;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = l;
        const int64_t x = r % la;
        r /= la;
        const int64_t y = r % lb;
        r /= lb;
        const int64_t i = r % li;
        const int64_t j = r / li;
        double v = a.t2[l];
        if (a.t1ai) v += a.t1ai[x + la * i] * a.t1bj[y + lb * j];
        if (a.t1aj) v -= a.t1aj[x + la * j] * a.t1bi[y + lb * i];
        a.tau[l] = v;
    }
}
__global__ void eri_gather_kernel(EriGatherArgs a, const double* __restrict__ eri) {
    const int64_t total = (int64_t)a.len[0] * a.len[1] * a.len[2] * a.len[3];
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < total; l += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = l, dst = a.off;
        int64_t g[4];
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const int x = (int)(r % a.len[p]);
            r /= a.len[p];
            dst += a.st[p] * x;
            g[p] = a.g[p][x];
        }
        const int64_t src = ((g[a.pos[0]] * a.n + g[a.pos[1]]) * a.n + g[a.pos[2]]) * a.n + g[a.pos[3]];
        a.C[dst] += a.sign * eri[src];
    }
}

}  // namespace

void eri_gather(const EriGatherArgs& a, const double* eri, cudaStream_t s) {
    const int64_t n = (int64_t)a.len[0] * a.len[1] * a.len[2] * a.len[3];
    if (n <= 0) return;
    eri_gather_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(a, eri);
    COUNT_LAUNCH();
}

namespace {
__global__ void closed_shell_jk_kernel(const double* __restrict__ eri, int n, int nocc, double* __restrict__ F) {
    const int64_t pq = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (pq >= (int64_t)n * n) return;
    const int64_t p = pq / n, q = pq % n, n2 = (int64_t)n * n, n3 = n2 * n;
    double v = 0;
    for (int i = 0; i < nocc; i++) v += 2.0 * eri[p * n3 + q * n2 + (int64_t)i * n + i] - eri[p * n3 + (int64_t)i * n2 + (int64_t)i * n + q];
    F[pq] = v;
}
}  // namespace

void closed_shell_jk(const double* eri, int n, int nocc, double* F, cudaStream_t s) {
    const int64_t nn = (int64_t)n * n;
    if (nn <= 0) return;
    closed_shell_jk_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(eri, n, nocc, F);
    COUNT_LAUNCH();
}

void tau_block(const TauArgs& a, cudaStream_t s) {
    const int64_t n = a.len[0] * a.len[1] * a.len[2] * a.len[3];
    if (n <= 0) return;
    tau_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(a);
    COUNT_LAUNCH();
}

void pack_vvvv(double* V, int kind_ab, int kind_cd, int n0, int n1, int n2, int n3, int64_t scd, const double* tJ,
               const double* tK, int a0, int a1, bool J, bool K, cudaStream_t s) {
    int64_t ncd = kind_cd == 1 ? (int64_t)n2 * (n2 - 1) / 2 : (int64_t)n2 * n3;
    int64_t total = (int64_t)(a1 - a0) * n1 * ncd;
    if (total <= 0) return;
    pack_vvvv_kernel<<<ew_blocks(total), EW_THREADS, 0, s>>>(V, kind_ab, kind_cd, n0, n1, n2, n3, scd, tJ, tK, a0,
                                                              a1, J, K);
    COUNT_LAUNCH();
}

void diis_advance(int* state, int order, cudaStream_t s) {
    diis_advance_kernel<<<1, 1, 0, s>>>(state, order);
    COUNT_LAUNCH();
}

void diis_store(const int* state, const double* const* xs, const double* const* dxs, const double* t1, int64_t n1,
                const double* t2, int64_t n2, const double* z1, const double* z2, cudaStream_t s) {
    diis_store_kernel<<<ew_blocks(n1 + n2), EW_THREADS, 0, s>>>(state, xs, dxs, t1, n1, t2, n2, z1, z2);
    COUNT_LAUNCH();
}

void diis_dots(const int* state, const double* const* dxs, int order, int64_t off, int64_t len, double w,
               double* dots, cudaStream_t s) {
    if (len <= 0) return;
    int nb = ew_blocks(len);
    double* part = partial_buffer(s);
    diis_dots_kernel<<<nb, EW_THREADS, 0, s>>>(state, dxs, order, off, len, part);
    fold_batch_kernel<<<1, 1024, 0, s>>>(part, nb, order, w, dots);
    COUNT_LAUNCH();
    COUNT_LAUNCH();
}

void diis_solve(int* state, double* e, double* c, const double* dots, int order, cudaStream_t s) {
    diis_solve_kernel<<<1, 32, 0, s>>>(state, e, c, dots, order);
    COUNT_LAUNCH();
}

void diis_store_segment(const int* state, const double* const* xs, const double* const* dxs, int64_t off,
                        const double* x, const double* dx, int64_t len, cudaStream_t s) {
    if (len <= 0) return;
    diis_store_segment_kernel<<<ew_blocks(len), EW_THREADS, 0, s>>>(state, xs, dxs, off, x, dx, len);
    COUNT_LAUNCH();
}

void lincomb_segment(double* out, int64_t len, const double* const* xs, int64_t off, const double* c, int nx,
                     cudaStream_t s) {
    if (len <= 0) return;
    lincomb_segment_kernel<<<ew_blocks(len), EW_THREADS, 0, s>>>(out, len, xs, off, c, nx);
    COUNT_LAUNCH();
}

void diis_damp(const int* state, const double* const* xs, int order, int64_t len, double damping, cudaStream_t s) {
    if (len <= 0 || damping <= 0.0) return;
    diis_damp_kernel<<<ew_blocks(len), EW_THREADS, 0, s>>>(state, xs, order, len, damping);
    COUNT_LAUNCH();
}

}  // namespace kern
}  // namespace ccsd
