// Split (Ozaki-style) contraction path on the sm_100a tensor cores.
//
// Each FP64 operand row x (a row of A(m,:) or a column of B(:,n), gathered through
// the planner's offset tables) is scaled by a power of two from its max-abs and cut
// into slices, round-to-nearest at each step (so the truncation error is unbiased):
//
// BF16 slices (3 or 4):   x = 2^(e-6) * (s1 + s2 + s3 [+ s4]),  2^e <= max|x| < 2^(e+1),
//   s1 an integer in [-128,128], s2 = integer/2^8, s3 = integer/2^16, all exact in BF16.
//   The tcgen05 GEMM (kind::f16) keeps FP32 accumulators in TMEM:
//     L2  = sum_k s1a*s1b                         (products <= 2^14: a chunk of 1024 k
//                                                    sums exactly in FP32)
//     L34 = the other products with i+j < NS      (2^-8 smaller)
//   and every chunk is drained into FP64 registers, so the leading term is exact and the
//   FP32 rounding of the rest sits ~2^-32 below the result (3 slices; 4 slices also keep
//   s1*s2 + s2*s1 apart, exact over 512 k).
//
// INT8 slices (3, 4 or 5):  x = (max/127) * (q1 + q2/254 + q3/254^2 ...),  q_t in [-127,127],
//   the whole signed 8-bit range: y = x * 127/max lies in [-127,127]; q1 = rint(y) and each
//   further slice is rint of the remainder (in [-1/2,1/2]) times 254, so every slice
//   carries log2(254) = 7.99 bits.  The tcgen05 GEMM (kind::i8, twice the BF16 rate)
//   accumulates every level t = i+j of the kept products q_i*q_j (i+j < NS) in its own
//   INT32 accumulator, which is exact (|q_i q_j| <= 127^2 < 2^14, at most 5 products per
//   level: a drained chunk of 16384 k stays below 2^31); the epilogue weights level t by
//   254^-t in FP64.  Per product the error is ~254^-NS / 2 of row max x column max
//   (3.7e-8, 1.5e-10, 5.7e-13 for 3, 4, 5 slices).
//
// Kernel structure (one 128 x TBN output tile per CTA, 320 threads):
//   warp 0      TMA producer: NS A-slice + NS B-slice tiles of 128-byte k-blocks per
//               stage (128-byte swizzle), 2 stages, mbarrier full/empty ring;
//   warp 1      TMEM allocation and the single-thread MMA issuer: one MMA per kept slice
//               product per k-step, commit to release smem stages and to publish a
//               finished chunk;
//   warps 2..9  epilogue: TMEM accumulator sets (double-buffered where two fit) are
//               drained per chunk into FP64 registers; the scaled result is scattered
//               into the destination through the planner's offset tables at the end.
// Every mbarrier wait is bounded (about 2 s); on expiry the kernel records an error
// code, stops issuing work and returns after releasing its TMEM.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace ccsd {
namespace kern {

extern std::atomic<int64_t> g_launches;
double* partial_buffer(cudaStream_t s);
void set_smem_once(const void* kernel, int bytes);

namespace split {

constexpr int BM = 128;
constexpr int EPI_WARPS = 8;
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr long long WAIT_CYCLES = 4000000000ll;     // ~2 s at 1.9 GHz
constexpr int SMEM_LIMIT = 227 * 1024;

// Kernel shape per scheme.  A stage holds NS A tiles and NS B tiles of one k-block (a
// 128- or 64-byte row segment); as many stages as fit in shared memory (at most 4).
template <int NS, bool I8>
struct Shape {
    // 4 and 5 INT8 slices use 64-byte k-blocks so that wider tiles still fit
    static constexpr int KBB = (I8 && NS >= 4) ? 64 : 128;          // bytes per k-block row
    static constexpr int BKE = KBB / (I8 ? 1 : 2);                  // k elements per k-block
    static constexpr int TBN = I8 ? (NS <= 4 ? 128 : 64) : (NS == 3 ? 128 : 64);
    static constexpr int TILE_A = BM * KBB;
    static constexpr int TILE_B = TBN * KBB;
    static constexpr int STAGE = NS * (TILE_A + TILE_B);
    static constexpr int STAGES_FIT = (SMEM_LIMIT - 1024 - 256) / STAGE;
    static constexpr int STAGES = STAGES_FIT < 4 ? STAGES_FIT : 4;
    static constexpr int KSTEPS = KBB / 32;                         // MMAs of 32 bytes of K per k-block
    // accumulators per buffer.  BF16: s1*s1 (exact over 1024 k) and the rest; 4 slices
    // also keep s1*s2 + s2*s1 apart (exact over 512 k).  INT8: one exact INT32
    // accumulator per level i+j.
    static constexpr int NACC = I8 ? NS : (NS == 4 ? 3 : 2);
    // k-blocks per drained chunk: 1024 / 512 k (BF16), 16384 k (INT8: |level| < 2^31)
    static constexpr int CHUNK = I8 ? 16384 / BKE : (NS == 4 ? 8 : 16);
    // split-K ranges: whole exact chunks (BF16), any 1024 k (INT8: exact per range)
    static constexpr int KSPLIT_GRAIN = I8 ? 1024 / BKE : CHUNK;
    static constexpr int BUF = NACC * TBN;                          // TMEM columns per buffer
    static constexpr int NBUF = 2 * BUF <= 512 ? 2 : 1;             // double-buffered if two fit
    static constexpr int TMEM_COLS = NBUF * BUF <= 256 ? 256 : 512;
    static constexpr int COLS = TBN / 2;                            // columns per epilogue warp
    static constexpr size_t SMEM = 1024 + (size_t)STAGES * STAGE + 256;
    // instruction descriptor: D = F32 / S32, A = B = BF16 / signed 8-bit, K-major both,
    // N = TBN, M = 128
    static constexpr uint32_t IDESC = (I8 ? (2u << 4) : (1u << 4)) | (1u << 7) | (1u << 10) |
                                      ((uint32_t)(TBN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
    static_assert(STAGES >= 2, "two stages must fit");
    static_assert(SMEM <= SMEM_LIMIT, "stages exceed shared memory");
    static_assert(BUF <= 512, "accumulators exceed TMEM");
    static_assert(TBN % 16 == 0 && TBN >= 16 && TBN <= 256, "MMA N");
};

struct Params {
    int M, N, K;
    int Mp, Np, Kp;
    int tiles_n;
    double alpha;
    const double* scaleA;
    const double* scaleB;
    double* C;
    const int64_t* Cm0;
    const int64_t* Cm1;
    const int64_t* Cn0;
    const int64_t* Cn1;
    int nvm, nvn;
    double vsign[4];
    int* err;
    // split-K over gridDim.y: K-block range blockIdx.y of ks, partials (scales applied,
    // alpha not) to ws[z][m][n], folded into C by the FP64 fold kernel
    int ks;
    int kb_per;                    // K blocks per range (a multiple of the exact chunk)
    double* ws;
    int dense;                     // write ws[z][m][n] even without split-K (merged products)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait; false on expiry (the error code is recorded and the abort flag set)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                          int code) {
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (clock64() - t0 > WAIT_CYCLES) {
            *abort_flag = 1;
            atomicCAS(err, 0, code);
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// K-major swizzled tile descriptor: rows of KBB (128 or 64) bytes, 8-row groups 8*KBB
// bytes apart, swizzle of the row width
template <int KBB>
__device__ __forceinline__ uint64_t sdesc(const void* p) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_u32(p) >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                           // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((8 * KBB) >> 4) << 32;            // stride byte offset
    d |= (uint64_t)1 << 46;                           // descriptor version (sm_100)
    d |= (uint64_t)(KBB == 128 ? 2 : 4) << 61;        // SWIZZLE_128B / SWIZZLE_64B
    return d;
}

template <bool I8>
__device__ __forceinline__ void umma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    if constexpr (I8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
            "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
            "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
    }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int NS, bool I8>
__global__ void __launch_bounds__(THREADS, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Params p) {
    using Sh = Shape<NS, I8>;
    constexpr int NBUF = Sh::NBUF, STAGES = Sh::STAGES;
    constexpr int TBN = Sh::TBN, COLS = Sh::COLS;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* stages = smem;
    uint64_t* bars = (uint64_t*)(smem + (size_t)STAGES * Sh::STAGE);
    uint64_t* full = bars;                   // [STAGES]
    uint64_t* empty = bars + STAGES;         // [STAGES]
    uint64_t* tfull = bars + 2 * STAGES;     // [2]
    uint64_t* tempty = bars + 2 * STAGES + 2;   // [2]
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 4);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x;
    const int tm = tile / p.tiles_n, tn = tile % p.tiles_n;
    const int m0 = tm * BM, n0 = tn * TBN;
    // this CTA's K blocks [kb0, kb0 + nkb)
    const int kb0 = blockIdx.y * p.kb_per;
    const int nkb = max(0, min(p.Kp / Sh::BKE, kb0 + p.kb_per) - kb0);
    const int nchunks = (nkb + Sh::CHUNK - 1) / Sh::CHUNK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI_WARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Sh::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            for (int kb = 0; kb < nkb && !*abort_flag; kb++) {
                const int s = kb % STAGES;
                if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1, abort_flag, p.err, 1)) break;
                mbar_expect_tx(&full[s], Sh::STAGE);
                uint8_t* base = stages + (size_t)s * Sh::STAGE;
                // x = k-block start in elements: a multiple of 128 bytes
                for (int i = 0; i < NS; i++)
                    tma_load_2d(base + i * Sh::TILE_A, &tmA, (kb0 + kb) * Sh::BKE, i * p.Mp + m0, &full[s]);
                for (int i = 0; i < NS; i++)
                    tma_load_2d(base + NS * Sh::TILE_A + i * Sh::TILE_B, &tmB, (kb0 + kb) * Sh::BKE,
                                i * p.Np + n0, &full[s]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int kb = 0;
            for (int c = 0; c < nchunks && !*abort_flag; c++) {
                const int b = c % NBUF;
                if (c >= NBUF && !mbar_wait(&tempty[b], ((c / NBUF) - 1) & 1, abort_flag, p.err, 2)) break;
                tc_fence_after();
                const uint32_t dbase = tmem + b * Sh::BUF;
                const int kb_end = min(nkb, (c + 1) * Sh::CHUNK);
                bool first = true;
                bool ok = true;
                for (; kb < kb_end; kb++) {
                    const int s = kb % STAGES;
                    if (!mbar_wait(&full[s], (kb / STAGES) & 1, abort_flag, p.err, 3)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint8_t* base = stages + (size_t)s * Sh::STAGE;
                    uint64_t ad[NS], bd[NS];
#pragma unroll
                    for (int i = 0; i < NS; i++) {
                        ad[i] = sdesc<Sh::KBB>(base + i * Sh::TILE_A);
                        bd[i] = sdesc<Sh::KBB>(base + NS * Sh::TILE_A + i * Sh::TILE_B);
                    }
#pragma unroll
                    for (int kk = 0; kk < Sh::KSTEPS; kk++) {
                        // one MMA covers 32 bytes of K (16 BF16 or 32 INT8 values)
                        const uint64_t o = (uint64_t)(kk * 32) >> 4;
                        // slice products (i, t - i) with t < NS into accumulator t (INT8) or
                        // min(t, NACC - 1) (BF16)
                        bool fresh[Sh::NACC];
#pragma unroll
                        for (int j = 0; j < Sh::NACC; j++) fresh[j] = first;
#pragma unroll
                        for (int t = 0; t < NS; t++)
#pragma unroll
                            for (int i = 0; i <= t; i++) {
                                const int j = t < Sh::NACC - 1 ? t : Sh::NACC - 1;
                                umma<I8>(dbase + j * TBN, ad[i] + o, bd[t - i] + o, Sh::IDESC, fresh[j] ? 0u : 1u);
                                fresh[j] = false;
                            }
                        first = false;
                    }
                    umma_commit(&empty[s]);
                }
                if (!ok) break;
                umma_commit(&tfull[b]);
            }
        }
    } else {
        // ---------------- epilogue ----------------
        const int ew = warp - 2;
        const int q = warp & 3;          // TMEM lane quadrant this warp may access
        const int h = ew >> 2;           // column half
        double acc[COLS];
#pragma unroll
        for (int j = 0; j < COLS; j++) acc[j] = 0.0;
        bool ok = true;
        for (int c = 0; c < nchunks; c++) {
            const int b = c % NBUF;
            if (!mbar_wait(&tfull[b], (c / NBUF) & 1, abort_flag, p.err, 4)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + b * Sh::BUF + h * COLS;
#pragma unroll
            for (int j4 = 0; j4 < COLS / 16; j4++) {
                if constexpr (I8) {
                    // one level at a time (fewer live registers): level j weighs 254^-j
#pragma unroll
                    for (int j = 0; j < Sh::NACC; j++) {
                        uint32_t r[16];
                        tmem_ld16(base + j * TBN + j4 * 16, r);
                        tmem_wait_ld();
                        const double w = j == 0 ? 1.0 : j == 1 ? 1.0 / 254.0 : j == 2 ? 1.0 / 64516.0
                                       : j == 3 ? 1.0 / 16387064.0 : 1.0 / 4162314256.0;
#pragma unroll
                        for (int t = 0; t < 16; t++) acc[j4 * 16 + t] += (double)(int)r[t] * w;
                    }
                } else {
                    uint32_t r[Sh::NACC][16];
#pragma unroll
                    for (int j = 0; j < Sh::NACC; j++) tmem_ld16(base + j * TBN + j4 * 16, r[j]);
                    tmem_wait_ld();
#pragma unroll
                    for (int t = 0; t < 16; t++) {
                        double v = 0.0;
#pragma unroll
                        for (int j = 0; j < Sh::NACC; j++) v += (double)__uint_as_float(r[j][t]);
                        acc[j4 * 16 + t] += v;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[b]);
        }
        if (ok && (p.ks > 1 || p.dense)) {
            const int m = m0 + q * 32 + lane;
            if (m < p.M) {
                const double sa = p.scaleA[m];
                double* wz = p.ws + ((int64_t)blockIdx.y * p.M + m) * p.N;
#pragma unroll
                for (int j = 0; j < COLS; j++) {
                    const int n = n0 + h * COLS + j;
                    if (n < p.N) wz[n] = sa * p.scaleB[n] * acc[j];
                }
            }
        } else if (ok && p.nvm == 1 && p.nvn == 1) {
            // one destination per element: read EB destinations, then write them, so that
            // the read-modify-writes of a thread overlap instead of running one by one
            constexpr int EB = 8;
            const int m = m0 + q * 32 + lane;
            if (m < p.M) {
                const double sa = p.alpha * p.vsign[0] * p.scaleA[m];
                const int64_t cm0 = p.Cm0[m];
#pragma unroll
                for (int j0 = 0; j0 < COLS; j0 += EB) {
                    int64_t off[EB];
                    double old[EB];
#pragma unroll
                    for (int t = 0; t < EB; t++) {
                        const int n = n0 + h * COLS + j0 + t;
                        off[t] = n < p.N ? cm0 + p.Cn0[n] : -1;
                    }
#pragma unroll
                    for (int t = 0; t < EB; t++) old[t] = off[t] >= 0 ? p.C[off[t]] : 0.0;
#pragma unroll
                    for (int t = 0; t < EB; t++) {
                        const int n = n0 + h * COLS + j0 + t;
                        if (off[t] >= 0) p.C[off[t]] = old[t] + sa * p.scaleB[n] * acc[j0 + t];
                    }
                }
            }
        } else if (ok) {
            const int m = m0 + q * 32 + lane;
            if (m < p.M) {
                const double sa = p.alpha * p.scaleA[m];
                const int64_t cm0 = p.Cm0[m];
                const int64_t cm1 = p.nvm > 1 ? p.Cm1[m] : 0;
#pragma unroll
                for (int j = 0; j < COLS; j++) {
                    const int n = n0 + h * COLS + j;
                    if (n < p.N) {
                        const double v = sa * p.scaleB[n] * acc[j];
                        const int64_t cn0 = p.Cn0[n];
                        p.C[cm0 + cn0] += p.vsign[0] * v;
                        if (p.nvn > 1) p.C[cm0 + p.Cn1[n]] += p.vsign[1] * v;
                        if (p.nvm > 1) {
                            p.C[cm1 + cn0] += p.vsign[p.nvn] * v;
                            if (p.nvn > 1) p.C[cm1 + p.Cn1[n]] += p.vsign[3] * v;
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Sh::TMEM_COLS));
    }
}

// ---------------------------------------------------------------------------
// slicing: two passes over 32-row x 64-k tiles of the gathered operand.  A CTA walks
// tiles t = blockIdx.x, + gridDim.x, ... (t = row tile + tiles_r * k tile); the offset
// tables of the next tile load while the current tile's elements are in flight.
// ---------------------------------------------------------------------------
constexpr int SR = 32, SK = 64, STHREADS = 256, SPER = (SR * SK) / STHREADS;
constexpr int SLICE_CTAS = 148 * 6;   // resident at 6 CTAs per SM (40 registers, 18 KB)

// offset tables of tile t into buffer b (-1 past the operand)
__device__ __forceinline__ void slice_tables(const int64_t* __restrict__ R, const int64_t* __restrict__ Kt, int nrows,
                                             int K, int tiles_r, int64_t t, int64_t (*sR)[SR], int64_t (*sK)[SK],
                                             int b) {
    const int r0 = (int)(t % tiles_r) * SR;
    const int64_t k0 = (t / tiles_r) * SK;
    for (int i = threadIdx.x; i < SR; i += STHREADS) sR[b][i] = (r0 + i < nrows) ? R[r0 + i] : -1;
    for (int i = threadIdx.x; i < SK; i += STHREADS) sK[b][i] = (k0 + i < K) ? Kt[k0 + i] : -1;
}

// element i of this thread in a tile: KC (k contiguous) walks k fastest, else r
template <bool KC>
__device__ __forceinline__ void slice_rk(int i, int& r, int& k) {
    const int e = threadIdx.x + i * STHREADS;
    if (KC) {
        k = e % SK;
        r = e / SK;
    } else {
        r = e % SR;
        k = e / SR;
    }
}

// Tiles are handed out in order: the first to CTA blockIdx.x, then the next free tile
// from a counter (ctr, zeroed with the row maxima) to whichever CTA asks, so that the tiles
// in flight stay a compact range of the operand, as with one CTA per tile.
__device__ __forceinline__ int64_t next_tile(unsigned long long* ctr, int64_t* s_next) {
    if (threadIdx.x == 0) *s_next = (int64_t)gridDim.x + (int64_t)atomicAdd(ctr, 1ull);
    __syncthreads();
    return *s_next;
}

template <bool KC>
__global__ void __launch_bounds__(STHREADS, 6) rowmax_kernel(const double* __restrict__ X, const int64_t* __restrict__ R,
                                                          const int64_t* __restrict__ Kt, int nrows, int K, int tiles_r,
                                                          int64_t ntiles, unsigned long long* rowmax,
                                                          unsigned long long* ctr) {
    __shared__ int64_t sR[2][SR], sK[2][SK];
    __shared__ double red[STHREADS / 32][SR];
    __shared__ int64_t s_next;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int b = 0;
    if ((int64_t)blockIdx.x < ntiles) slice_tables(R, Kt, nrows, K, tiles_r, blockIdx.x, sR, sK, 0);
    __syncthreads();
    for (int64_t t = blockIdx.x, tn; t < ntiles; t = tn, b ^= 1) {
        double v[SPER];
#pragma unroll
        for (int i = 0; i < SPER; i++) {
            int r, k;
            slice_rk<KC>(i, r, k);
            const int64_t orr = sR[b][r], ok = sK[b][k];
            v[i] = (orr >= 0 && ok >= 0) ? fabs(X[orr + ok]) : 0.0;
        }
        tn = next_tile(ctr, &s_next);
        if (tn < ntiles) slice_tables(R, Kt, nrows, K, tiles_r, tn, sR, sK, b ^ 1);
        const int r0 = (int)(t % tiles_r) * SR;
        if (KC) {
            // element i of a warp: one row (warp / 2 + 4 i), 32 consecutive k
#pragma unroll
            for (int i = 0; i < SPER; i++) {
                double m = v[i];
                for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
                const int row = r0 + (warp >> 1) + 4 * i;
                if (lane == 0 && row < nrows && m > 0.0)
                    atomicMax(&rowmax[row], (unsigned long long)__double_as_longlong(m));
            }
        } else {
            // every element of a thread sits in row `lane`: fold them, then across the warps
            double m = 0.0;
#pragma unroll
            for (int i = 0; i < SPER; i++) m = fmax(m, v[i]);
            red[warp][lane] = m;
            __syncthreads();
            if (warp == 0) {
                for (int w = 1; w < STHREADS / 32; w++) m = fmax(m, red[w][lane]);
                const int row = r0 + lane;
                if (row < nrows && m > 0.0) atomicMax(&rowmax[row], (unsigned long long)__double_as_longlong(m));
            }
        }
        __syncthreads();   // next tables visible, red free again
    }
}

__device__ __forceinline__ unsigned short bf16_bits(double v) {
    __nv_bfloat16 b = __float2bfloat16_rn((float)v);
    return *reinterpret_cast<unsigned short*>(&b);
}

template <bool KC, int NS, bool I8>
__global__ void __launch_bounds__(STHREADS, 6)
    slice_kernel(const double* __restrict__ X, const int64_t* __restrict__ R, const int64_t* __restrict__ Kt, int nrows,
                 int K, int tiles_r, int64_t ntiles, const unsigned long long* __restrict__ rowmax, int rows_p, int kpad,
                 uint8_t* __restrict__ out_bytes, double* __restrict__ scale, unsigned long long* ctr) {
    __shared__ double tile[SR][SK + 1];
    __shared__ int64_t sR[2][SR], sK[2][SK];
    __shared__ double sMul[SR];      // per row: 127 / max (INT8) or 2^(6 - e) (BF16); 0 for a zero row
    __shared__ int64_t s_next;
    const size_t plane = (size_t)rows_p * kpad;
    int b = 0;
    if ((int64_t)blockIdx.x < ntiles) slice_tables(R, Kt, nrows, K, tiles_r, blockIdx.x, sR, sK, 0);
    __syncthreads();
    for (int64_t t = blockIdx.x, tn; t < ntiles; t = tn, b ^= 1) {
        const int r0 = (int)(t % tiles_r) * SR;
        const int64_t k0 = (t / tiles_r) * SK;
        double v[SPER];
#pragma unroll
        for (int i = 0; i < SPER; i++) {
            int r, k;
            slice_rk<KC>(i, r, k);
            const int64_t orr = sR[b][r], ok = sK[b][k];
            v[i] = (orr >= 0 && ok >= 0) ? X[orr + ok] : 0.0;
        }
        if (threadIdx.x < SR) {
            const int row = r0 + threadIdx.x;
            const double mx = row < nrows ? __longlong_as_double((long long)rowmax[row]) : 0.0;
            double mul = 0.0, sc = 0.0;
            if (mx > 1e-290) {   // below that a row counts as zero (127 / max would overflow)
                if constexpr (I8) {
                    mul = 127.0 / mx;
                    sc = mx / 127.0;
                } else {
                    mul = ldexp(1.0, 6 - ilogb(mx));          // mx in [2^e, 2^(e+1))
                    sc = ldexp(1.0, ilogb(mx) - 6);
                }
            }
            sMul[threadIdx.x] = mul;
            if (k0 == 0 && row < rows_p) scale[row] = sc;
        }
        tn = next_tile(ctr, &s_next);
        if (tn < ntiles) slice_tables(R, Kt, nrows, K, tiles_r, tn, sR, sK, b ^ 1);
#pragma unroll
        for (int i = 0; i < SPER; i++) {
            int r, k;
            slice_rk<KC>(i, r, k);
            tile[r][k] = v[i];
        }
        __syncthreads();
        // BF16: x = 2^(e-6) (s1 + s2 + ...), s1 in [-128,128], slice t carries weight 2^-8t
        // INT8: x = (max/127) (q1 + q2/254 + ...), q_t in [-127,127]
#pragma unroll
        for (int i = 0; i < SPER; i++) {
            const int e = threadIdx.x + i * STHREADS;
            const int k = e % SK, r = e / SK;
            const int row = r0 + r;
            const double mul = sMul[r];
            uint16_t bits[NS];
#pragma unroll
            for (int q = 0; q < NS; q++) bits[q] = 0;
            if (mul > 0.0) {
                double y = tile[r][k] * mul;                 // |y| <= 127 (INT8), < 2^7 + 1 (BF16)
                double w = 1.0;                              // BF16 weight of slice q: 2^(-8q)
#pragma unroll
                for (int q = 0; q < NS; q++) {
                    const double st = rint(y);               // an integer of at most 8 significant bits
                    if constexpr (I8) {
                        bits[q] = (uint16_t)(uint8_t)(int8_t)(int)st;
                        y = (y - st) * 254.0;                // remainder in [-1/2, 1/2] -> [-127, 127]
                    } else {
                        bits[q] = bf16_bits(st * w);
                        y = (y - st) * 256.0;
                        w *= 0.00390625;
                    }
                }
            }
            const size_t o = (size_t)row * kpad + (size_t)(k0 + k);
            if constexpr (I8) {
#pragma unroll
                for (int q = 0; q < NS; q++) out_bytes[q * plane + o] = (uint8_t)bits[q];
            } else {
                uint16_t* out = reinterpret_cast<uint16_t*>(out_bytes);
#pragma unroll
                for (int q = 0; q < NS; q++) out[q * plane + o] = bits[q];
            }
        }
        __syncthreads();   // the tile, sMul and the next tables
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)f;
    });
    return fn;
}

void make_map(CUtensorMap* map, const uint8_t* base, int kind, int rows_total, int kpad, int box_rows, int kbb) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) throw std::runtime_error("cuTensorMapEncodeTiled is not available");
    const int eb = slice_elem_bytes(kind);
    cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows_total};
    cuuint64_t strides[1] = {(cuuint64_t)kpad * eb};
    cuuint32_t box[2] = {(cuuint32_t)(kbb / eb), (cuuint32_t)box_rows};   // one k-block of kbb bytes
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, kind == SLICE_INT8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                     (void*)base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, kbb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

int* error_flag() {
    static std::mutex mu;
    static std::map<int, int*> flags;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = flags.find(dev);
    if (it != flags.end()) return it->second;
    int* f = nullptr;
    cudaMalloc(&f, sizeof(int));
    cudaMemset(f, 0, sizeof(int));
    flags[dev] = f;
    return f;
}

}  // namespace split

bool split_supported() {
    static const bool ok = [] {
        int dev = 0;
        cudaDeviceProp prop;
        return cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess &&
               prop.major == 10 && split::encode_fn() != nullptr;
    }();
    return ok;
}

int split_rows_pad(int rows) { return (rows + split::BM - 1) / split::BM * split::BM; }
int split_k_pad(int k, int kind) {
    const int bke = 128 / slice_elem_bytes(kind);   // a multiple of every scheme's k-block
    return (k + bke - 1) / bke * bke;
}

namespace {
template <int NS, bool I8>
void launch_slice(int grid, int tiles_r, int64_t ntiles, bool kcontig, const double* X, const int64_t* R,
                  const int64_t* Kt, int nrows, int K, const unsigned long long* rowmax, SlicedOperand& out,
                  cudaStream_t s) {
    using namespace split;
    unsigned long long* ctr = const_cast<unsigned long long*>(rowmax) + out.rows + 1;
    if (kcontig)
        slice_kernel<true, NS, I8><<<grid, STHREADS, 0, s>>>(X, R, Kt, nrows, K, tiles_r, ntiles, rowmax, out.rows,
                                                             out.kpad, out.data, out.scale, ctr);
    else
        slice_kernel<false, NS, I8><<<grid, STHREADS, 0, s>>>(X, R, Kt, nrows, K, tiles_r, ntiles, rowmax, out.rows,
                                                              out.kpad, out.data, out.scale, ctr);
}
}  // namespace

void slice_rows(const double* X, const int64_t* R, const int64_t* Kt, int nrows, int K, bool kcontig,
                SlicedOperand& out, cudaStream_t s) {
    using namespace split;
    const int ns = out.nslices;
    if (!slice_scheme_ok(out.kind, ns)) throw std::runtime_error("unsupported slice scheme");
    if ((int64_t)ns * out.rows * out.kpad * slice_elem_bytes(out.kind) > out.bytes)
        throw std::runtime_error("sliced operand smaller than its scheme needs");
    unsigned long long* rowmax = reinterpret_cast<unsigned long long*>(out.rowmax);
    // the row maxima and, after them, the tile counters of the two passes
    cudaMemsetAsync(rowmax, 0, sizeof(double) * (out.rows + 2), s);
    const int tiles_r = out.rows / SR;
    const int64_t ntiles = (int64_t)tiles_r * (out.kpad / SK);
    const int grid = (int)std::min<int64_t>(ntiles, SLICE_CTAS);
    if (kcontig) rowmax_kernel<true><<<grid, STHREADS, 0, s>>>(X, R, Kt, nrows, K, tiles_r, ntiles, rowmax, rowmax + out.rows);
    else rowmax_kernel<false><<<grid, STHREADS, 0, s>>>(X, R, Kt, nrows, K, tiles_r, ntiles, rowmax, rowmax + out.rows);
    if (out.kind == SLICE_INT8) {
        if (ns == 3) launch_slice<3, true>(grid, tiles_r, ntiles, kcontig, X, R, Kt, nrows, K, rowmax, out, s);
        else if (ns == 4) launch_slice<4, true>(grid, tiles_r, ntiles, kcontig, X, R, Kt, nrows, K, rowmax, out, s);
        else launch_slice<5, true>(grid, tiles_r, ntiles, kcontig, X, R, Kt, nrows, K, rowmax, out, s);
    } else {
        if (ns == 3) launch_slice<3, false>(grid, tiles_r, ntiles, kcontig, X, R, Kt, nrows, K, rowmax, out, s);
        else launch_slice<4, false>(grid, tiles_r, ntiles, kcontig, X, R, Kt, nrows, K, rowmax, out, s);
    }
    g_launches += 2;
}

namespace {
struct SchemeInfo {
    int tbn, bke, kbb, chunk, grain;
    size_t smem;
    const void* kfn;
};

template <int NS, bool I8>
SchemeInfo scheme_info() {
    using Sh = split::Shape<NS, I8>;
    return {Sh::TBN, Sh::BKE, Sh::KBB, Sh::CHUNK, Sh::KSPLIT_GRAIN, Sh::SMEM,
            (const void*)split::split_gemm_kernel<NS, I8>};
}

SchemeInfo scheme(int kind, int ns) {
    if (kind == SLICE_INT8) {
        if (ns == 3) return scheme_info<3, true>();
        if (ns == 4) return scheme_info<4, true>();
        if (ns == 5) return scheme_info<5, true>();
    } else {
        if (ns == 3) return scheme_info<3, false>();
        if (ns == 4) return scheme_info<4, false>();
    }
    throw std::runtime_error("unsupported slice scheme");
}
}  // namespace

int split_ksplit(int M, int N, int K, int nslices, int kind) {
    using namespace split;
    const SchemeInfo si = scheme(kind, nslices);
    const int64_t tiles = (int64_t)((M + BM - 1) / BM) * ((N + si.tbn - 1) / si.tbn);
    if (tiles >= 148) return 1;
    const int64_t grains = (split_k_pad(K, kind) / si.bke + si.grain - 1) / si.grain;
    int64_t ks = (2 * 148 + tiles - 1) / tiles;
    ks = std::min<int64_t>(ks, grains);
    ks = std::min<int64_t>(ks, 256);
    return (int)std::max<int64_t>(ks, 1);
}

void gemm_split(const SlicedOperand& a, const SlicedOperand& b, int M, int N, int K, const GemmArgs& g,
                cudaStream_t s, int ks) {
    using namespace split;
    (void)K;
    const int ns = a.nslices, kind = a.kind;
    if (b.nslices != ns || b.kind != kind || a.kpad != b.kpad)
        throw std::runtime_error("split GEMM operands sliced differently");
    const SchemeInfo si = scheme(kind, ns);
    set_smem_once(si.kfn, (int)si.smem);
    CUtensorMap ma, mb;
    make_map(&ma, a.data, kind, ns * a.rows, a.kpad, BM, si.kbb);
    make_map(&mb, b.data, kind, ns * b.rows, b.kpad, si.tbn, si.kbb);
    Params p;
    p.M = M;
    p.N = N;
    p.K = K;
    p.Mp = a.rows;
    p.Np = b.rows;
    p.Kp = a.kpad;
    p.tiles_n = b.rows / si.tbn;
    p.alpha = g.alpha;
    p.scaleA = a.scale;
    p.scaleB = b.scale;
    p.C = g.C;
    p.Cm0 = g.Cm[0];
    p.Cm1 = g.Cm[1];
    p.Cn0 = g.Cn[0];
    p.Cn1 = g.Cn[1];
    p.nvm = g.nvm;
    p.nvn = g.nvn;
    for (int i = 0; i < 4; i++) p.vsign[i] = g.vsign[i];
    p.err = error_flag();
    const int nkb = a.kpad / si.bke;
    if (ks > 1 && (!g.ws || (int64_t)ks * M * N > g.ws_elems)) ks = 1;
    if (ks > 65535) ks = 65535;
    // K blocks per range: whole grains
    const int per_grains = ((nkb + si.grain - 1) / si.grain + ks - 1) / ks;
    p.ks = ks;
    p.kb_per = ks > 1 ? per_grains * si.grain : nkb;
    p.ws = g.ws;
    p.dense = g.dense_out ? 1 : 0;
    if (g.dense_out && (!g.ws || (int64_t)ks * M * N > g.ws_elems))
        throw std::runtime_error("merged split product: dense output workspace too small");
    const int tiles = (a.rows / BM) * p.tiles_n;
    const dim3 grid(tiles, ks);
    if (kind == SLICE_INT8) {
        if (ns == 3) split_gemm_kernel<3, true><<<grid, THREADS, si.smem, s>>>(ma, mb, p);
        else if (ns == 4) split_gemm_kernel<4, true><<<grid, THREADS, si.smem, s>>>(ma, mb, p);
        else split_gemm_kernel<5, true><<<grid, THREADS, si.smem, s>>>(ma, mb, p);
    } else {
        if (ns == 3) split_gemm_kernel<3, false><<<grid, THREADS, si.smem, s>>>(ma, mb, p);
        else split_gemm_kernel<4, false><<<grid, THREADS, si.smem, s>>>(ma, mb, p);
    }
    g_launches++;
    if (ks > 1 && !g.dense_out) splitk_fold(g, ks, s);
}

// ---------------------------------------------------------------------------
// merged symmetry-blocked products: slicing of rectangles of a merged operand, and the
// scatter of the merged dense product into the blocks of C
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ int find_rect(const int64_t* __restrict__ ts, int n, int64_t t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ts[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// one 32 x 64 tile of one rectangle per CTA: element (r, k) of the rectangle into v (0
// outside), lanes along k where the rectangle's k are contiguous, else along the rows
__device__ __forceinline__ void rect_tile(const RectDesc& d, int64_t lt, int& r0, int& k0, double* v, int64_t* sR,
                                          int64_t* sK) {
    using namespace split;
    r0 = (int)(lt % d.tiles_r) * SR;
    k0 = (int)(lt / d.tiles_r) * SK;
    for (int i = threadIdx.x; i < SR; i += STHREADS) sR[i] = (r0 + i < d.nrows) ? d.R[r0 + i] : -1;
    for (int i = threadIdx.x; i < SK; i += STHREADS) sK[i] = (k0 + i < d.nk) ? d.Kt[k0 + i] : -1;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SPER; i++) {
        const int e = threadIdx.x + i * STHREADS;
        const int r = d.kc ? e / SK : e % SR, k = d.kc ? e % SK : e / SR;
        v[i] = (sR[r] >= 0 && sK[k] >= 0) ? d.mul * d.X[sR[r] + sK[k]] : 0.0;
    }
}

// A CTA takes RECT_TPC consecutive tiles: one binary search over the rectangles' first
// tiles, then a forward walk (a batched launch covers some 10^5 rectangles, and a search
// per tile was a chain of 17 dependent loads in front of 16 KB of work)
constexpr int RECT_TPC = 8;

__device__ __forceinline__ int next_rect(const int64_t* __restrict__ ts, int n, int sp, int64_t t, bool first) {
    if (first) return find_rect(ts, n, t);
    while (sp + 1 < n && ts[sp + 1] <= t) sp++;
    return sp;
}

__global__ void __launch_bounds__(split::STHREADS) rect_rowmax_kernel(const RectDesc* __restrict__ rd,
                                                                      const int64_t* __restrict__ ts, int n,
                                                                      int64_t ntiles, unsigned long long* rowmax) {
    using namespace split;
    __shared__ int64_t sR[SR], sK[SK];
    __shared__ double red[STHREADS / 32][SR];
    __shared__ int sp;
    const int64_t t0 = (int64_t)blockIdx.x * RECT_TPC;
    const int64_t t1 = t0 + RECT_TPC < ntiles ? t0 + RECT_TPC : ntiles;
    for (int64_t t = t0; t < t1; t++) {
        if (threadIdx.x == 0) sp = next_rect(ts, n, sp, t, t == t0);
        __syncthreads();
        const RectDesc& d = rd[sp];
        unsigned long long* rm = d.rowmax ? d.rowmax : rowmax;
        int r0, k0;
        double v[SPER];
        rect_tile(d, t - ts[sp], r0, k0, v, sR, sK);
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (d.kc) {
#pragma unroll
            for (int i = 0; i < SPER; i++) {
                double m = fabs(v[i]);
                for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
                const int r = (warp >> 1) + 4 * i;
                if (lane == 0 && r0 + r < d.nrows && m > 0.0)
                    atomicMax(&rm[d.row0 + r0 + r], (unsigned long long)__double_as_longlong(m));
            }
        } else {
            double m = 0.0;
#pragma unroll
            for (int i = 0; i < SPER; i++) m = fmax(m, fabs(v[i]));
            red[warp][lane] = m;
            __syncthreads();
            if (warp == 0) {
                for (int w = 1; w < STHREADS / 32; w++) m = fmax(m, red[w][lane]);
                if (r0 + lane < d.nrows && m > 0.0)
                    atomicMax(&rm[d.row0 + r0 + lane], (unsigned long long)__double_as_longlong(m));
            }
        }
        __syncthreads();   // the tables and the reduction slots are reused by the next tile
    }
}

template <int NS>
__global__ void __launch_bounds__(split::STHREADS) rect_slice_kernel(const RectDesc* __restrict__ rd,
                                                                     const int64_t* __restrict__ ts, int n,
                                                                     int64_t ntiles, const unsigned long long* rowmax0,
                                                                     int rows_p0, int kpad0, uint8_t* out0,
                                                                     double* scale0) {
    using namespace split;
    __shared__ double tile[SR][SK + 1];
    __shared__ int64_t sR[SR], sK[SK];
    __shared__ double sMul[SR];
    __shared__ int sp;
    const int64_t t0 = (int64_t)blockIdx.x * RECT_TPC;
    const int64_t t1 = t0 + RECT_TPC < ntiles ? t0 + RECT_TPC : ntiles;
    for (int64_t t = t0; t < t1; t++) {
        if (threadIdx.x == 0) sp = next_rect(ts, n, sp, t, t == t0);
        __syncthreads();
        const RectDesc& d = rd[sp];
        // the rectangle's own merged operand, or the launch's
        const unsigned long long* rowmax = d.out ? d.rowmax : rowmax0;
        const int rows_p = d.out ? d.rows_p : rows_p0, kpad = d.out ? d.kpad : kpad0;
        uint8_t* out = d.out ? d.out : out0;
        double* scale = d.out ? d.scale : scale0;
        int r0, k0;
        double v[SPER];
        rect_tile(d, t - ts[sp], r0, k0, v, sR, sK);
        if (threadIdx.x < SR) {
            const int row = d.row0 + r0 + threadIdx.x;
            const bool in = r0 + (int)threadIdx.x < d.nrows;
            const double mx = in ? __longlong_as_double((long long)rowmax[row]) : 0.0;
            const bool nz = mx > 1e-290;
            sMul[threadIdx.x] = nz ? 127.0 / mx : 0.0;
            if (in && d.k0 == 0 && k0 == 0) scale[row] = nz ? mx / 127.0 : 0.0;   // the row's first rectangle
        }
#pragma unroll
        for (int i = 0; i < SPER; i++) {
            const int e = threadIdx.x + i * STHREADS;
            const int r = d.kc ? e / SK : e % SR, k = d.kc ? e % SK : e / SR;
            tile[r][k] = v[i];
        }
        __syncthreads();
        const size_t plane = (size_t)rows_p * kpad;
#pragma unroll
        for (int i = 0; i < SPER; i++) {
            const int e = threadIdx.x + i * STHREADS;
            const int k = e % SK, r = e / SK;
            if (r0 + r >= d.nrows || k0 + k >= d.nk) continue;
            const double mul = sMul[r];
            const size_t o = (size_t)(d.row0 + r0 + r) * kpad + (size_t)(d.k0 + k0 + k);
            double y = tile[r][k] * mul;
#pragma unroll
            for (int q = 0; q < NS; q++) {
                const double st = mul > 0.0 ? rint(y) : 0.0;
                out[q * plane + o] = (uint8_t)(int8_t)(int)st;
                y = (y - st) * 254.0;
            }
        }
        __syncthreads();   // the tile, the tables and the row factors are reused by the next tile
    }
}

// C[Cm_a[m] + Cn_b[n]] += vsign_ab * alpha * sum_z ws[z][row0 + m][col0 + n] for one
// rectangle's chunk of kBatchChunk elements per CTA
__global__ void __launch_bounds__(256) rect_scatter_kernel(const ScatterDesc* __restrict__ sd,
                                                           const int64_t* __restrict__ cs, int n,
                                                           const double* __restrict__ ws, int ldn, int64_t zstride,
                                                           int ks) {
    __shared__ int sp;
    if (threadIdx.x == 0) sp = find_rect(cs, n, blockIdx.x);
    __syncthreads();
    const ScatterDesc& d = sd[sp];
    const int64_t base = (blockIdx.x - cs[sp]) * (int64_t)kBatchChunk;
    const int64_t total = (int64_t)d.nrows * d.ncols;
    for (int i = threadIdx.x; i < kBatchChunk; i += blockDim.x) {
        const int64_t l = base + i;
        if (l >= total) break;
        const int m = (int)(l / d.ncols), c = (int)(l % d.ncols);
        const int64_t w = (int64_t)(d.row0 + m) * ldn + d.col0 + c;
        double v = 0.0;
        for (int z = 0; z < ks; z++) v += ws[z * zstride + w];
        v *= d.alpha;
        for (int a = 0; a < d.nvm; a++)
            for (int b = 0; b < d.nvn; b++) d.C[d.Cm[a][m] + d.Cn[b][c]] += d.vsign[a * d.nvn + b] * v;
    }
}

}  // namespace

void rect_slice(const RectDesc* d, const int64_t* tile_start, int n, int64_t ntiles, int ns, SlicedOperand& out,
                cudaStream_t s) {
    using namespace split;
    if (n <= 0 || ntiles <= 0) return;
    if (out.kind != SLICE_INT8) throw std::runtime_error("merged products slice to INT8 only");
    unsigned long long* rowmax = reinterpret_cast<unsigned long long*>(out.rowmax);
    cudaMemsetAsync(rowmax, 0, sizeof(double) * out.rows, s);
    cudaMemsetAsync(out.scale, 0, sizeof(double) * out.rows, s);
    cudaMemsetAsync(out.data, 0, (size_t)ns * out.rows * out.kpad, s);
    const unsigned grid = (unsigned)((ntiles + RECT_TPC - 1) / RECT_TPC);
    rect_rowmax_kernel<<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, rowmax);
    if (ns == 3) rect_slice_kernel<3><<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, rowmax, out.rows, out.kpad, out.data, out.scale);
    else if (ns == 4) rect_slice_kernel<4><<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, rowmax, out.rows, out.kpad, out.data, out.scale);
    else rect_slice_kernel<5><<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, rowmax, out.rows, out.kpad, out.data, out.scale);
    g_launches += 2;
}

void rect_slice_batched(const RectDesc* d, const int64_t* tile_start, int n, int64_t ntiles, int ns,
                        void* rowmax_arena, size_t rowmax_bytes, cudaStream_t s) {
    using namespace split;
    if (n <= 0 || ntiles <= 0) return;
    cudaMemsetAsync(rowmax_arena, 0, rowmax_bytes, s);
    const unsigned grid = (unsigned)((ntiles + RECT_TPC - 1) / RECT_TPC);
    rect_rowmax_kernel<<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, nullptr);
    if (ns == 3) rect_slice_kernel<3><<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, nullptr, 0, 0, nullptr, nullptr);
    else if (ns == 4) rect_slice_kernel<4><<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, nullptr, 0, 0, nullptr, nullptr);
    else rect_slice_kernel<5><<<grid, STHREADS, 0, s>>>(d, tile_start, n, ntiles, nullptr, 0, 0, nullptr, nullptr);
    g_launches += 2;
}

void rect_scatter(const ScatterDesc* d, const int64_t* chunk_start, int n, int64_t chunks, const double* ws, int ldn,
                  int64_t zstride, int ks, cudaStream_t s) {
    if (n <= 0 || chunks <= 0) return;
    rect_scatter_kernel<<<(unsigned)chunks, 256, 0, s>>>(d, chunk_start, n, ws, ldn, zstride, ks);
    g_launches++;
}

int split_error(bool reset) {
    int* f = split::error_flag();
    int h = 0;
    cudaMemcpy(&h, f, sizeof(int), cudaMemcpyDeviceToHost);
    if (reset && h) cudaMemset(f, 0, sizeof(int));
    return h;
}

}  // namespace kern
}  // namespace ccsd
