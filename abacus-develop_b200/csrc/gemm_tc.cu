// Complex FP32 GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32) with
// split precision: every FP32 operand x is split into hi = tf32(x) (rounded) and
// lo = x - hi, and C = A_hi*B_hi + A_hi*B_lo + A_lo*B_hi is accumulated in FP32 in
// tensor memory (the hi/lo "3xTF32" scheme: about FP32 accuracy at tensor-core rate).
//
//   C (M x N, column-major, complex) = alpha * op(A) * B + beta * C
//   op(A) = A   (A column-major M x K)            "N"
//   op(A) = A^H (A column-major K x M)            "C"
//   B column-major K x N.
//
// The complex product is done as one real GEMM of size 2M x N x 2K: with
// interleaved (re, im) storage B is already the real 2K x N matrix, and op(A)
// becomes the real 2M x 2K matrix whose 2x2 blocks are [[ar, -ai], [ai, ar]]
// (for A^H: [[ar, ai], [-ai, ar]]).  That expanded operand lives in tensor memory:
// the TMA-loaded raw tile of A (a column of A per 128-byte row for "N", MN-major; a
// row of A^H for "C", K-major) is read from shared memory by the epilogue warps, one
// real row of op(A) per thread, split into hi/lo and written to TMEM with tcgen05.st,
// and tcgen05.mma reads A from TMEM and only B from shared memory.  B is split in
// shared memory (hi in place, lo beside it), or, when many M tiles read it, once per
// call in HBM (k_split_b) so that the CTAs only copy it.
//
// CTA: 10 warps.  warp 0 issues TMA loads (cp.async.bulk.tensor, no multicast),
// warp 1 allocates TMEM (512 columns: two accumulators + one expanded A tile per
// stage) and one lane issues tcgen05.mma, warps 2-9 split/expand the tiles, drain
// TMEM and run the epilogue (alpha/beta -> global).
// 4-stage mbarrier pipeline, two TMEM accumulators.  Every wait is bounded in time; a wait that runs out
// sets an error word, the CTA drains its own copies in flight, frees TMEM and
// returns.  Long K is split across CTAs (grid.z) with a deterministic reduction.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>

#include "common.h"
#include "gemm_tc.h"
#include "tcgen05_util.cuh"

namespace b200 {
namespace {

using namespace tcu;

constexpr int kBM = 128;     // real rows of C per tile
constexpr int kBK = 32;      // real K per stage (one 128-byte swizzle row of fp32)
constexpr int kStages = 4;
constexpr int kAcc = 2;      // K stages accumulated in one TMEM buffer before it is drained
constexpr int kThreads = 320;   // warp 0 TMA, warp 1 MMA, warps 2-9 split / drain / store

// D (TMEM) (+)= A (TMEM: M = 128 rows in lanes 0..127, one column per K element) * B (shared-memory descriptor)
__device__ __forceinline__ void mma_tf32_ta(unsigned tmem_d, unsigned tmem_a, unsigned long long b, unsigned idesc,
                                            unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float* v) {
    unsigned r[16];
    // load and wait in one statement: the destination registers are only valid after tcgen05.wait::ld
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive TMEM columns of this thread's lane (warp w may access lanes 32 (w % 4) .. +31)
__device__ __forceinline__ void tmem_st16(unsigned taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::
            "r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// hi part of the split: x rounded to the nearest TF32 value (10 explicit mantissa bits); lo = x - hi is exact
__device__ __forceinline__ float tf32_round(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
// physical byte offset of (row, 16-byte chunk) in a 1024-byte-aligned SW128 tile with 128-byte rows
__device__ __forceinline__ unsigned sw128(unsigned row, unsigned chunk) {
    return row * 128u + ((chunk ^ (row & 7u)) << 4);
}
// per stage in shared memory: the raw A tile, then B (rounded hi in place, or the pre-split hi), then B lo
template <int BN> struct TileBytes {
    static constexpr int a_raw = 8192;   // 64 rows x 128 B ("C")  or 4 x 16 x 128 B ("N")
    static constexpr int b = BN * 128;
    static constexpr int stage = a_raw + 2 * b;
    static constexpr int need = kStages * stage + 2048;  // + barriers / flags + 1024-byte alignment slack
    // at least 120 KB, so that one CTA holds an SM and its 512 TMEM columns
    static constexpr int total = need > 120 * 1024 ? need : 120 * 1024;
};

// TMEM columns: two accumulators [0, 2 BN), then per stage s the expanded A tile at 2 BN + 64 s: hi in
// columns [0, 32), lo in [32, 64) (one column per real K, one lane per real row of C)
template <int BN> constexpr unsigned a_col(int s) { return unsigned(2 * BN + 64 * s); }
static_assert(2 * 128 + 64 * kStages <= 512, "TMEM columns");

// OPA: 0 = "N" (A column-major M x K, MN-major tiles), 1 = "C" (A^H of a column-major K x M, K-major tiles)
// PRE: B arrives already split (hi and lo tiles from HBM, written once per call by k_split_b)
//
// Accumulation: the tensor-core accumulator truncates on every accumulate, so a long
// chain of MMAs into one TMEM accumulator drifts (about 2e-8 relative per MMA).  Every
// kAcc K stages (24 MMAs) therefore start a fresh accumulator in one of two TMEM buffers;
// the epilogue warps drain the finished buffer into FP32 registers (IEEE round-to-nearest
// adds) while the next group runs in the other buffer.
template <int BN, int OPA, int PRE>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_cgemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
               const __grid_constant__ CUtensorMap mapBl, int M2, int N, int K2, int kstages_per_split, float2 alpha,
               float2 beta, float* __restrict__ C, long ldc2, float* __restrict__ ws, int* __restrict__ err,
               unsigned long long wait_ns) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // pipeline waits use wait_ns; the waits for this CTA's own copies and MMAs in flight after an abort use
    // at least the default, as they always end (plain loads of valid memory, MMAs on resident operands)
    const unsigned long long drain_ns = wait_ns > kWaitNs ? wait_ns : kWaitNs;
    using TB = TileBytes<BN>;
    // 1024-byte alignment of the tile area (the swizzle pattern depends on address bits 7..9)
    unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    unsigned char* bars = base + kStages * TB::stage;
    unsigned long long* full = reinterpret_cast<unsigned long long*>(bars);
    unsigned long long* ready = full + kStages;
    unsigned long long* empty = ready + kStages;
    unsigned long long* acc_full = empty + kStages;   // [2] MMA -> epilogue: stage result in TMEM buffer b
    unsigned long long* acc_empty = acc_full + 2;     // [2] epilogue -> MMA: buffer b drained
    unsigned* tmem_slot = reinterpret_cast<unsigned*>(acc_empty + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // "N": the N tile is the fastest grid index, so the few CTAs that read one A tile run together and
    // A crosses HBM once; "C": the M tile is, for the same reason with B
    const int tile_m = OPA == 0 ? blockIdx.y : blockIdx.x, tile_n = OPA == 0 ? blockIdx.x : blockIdx.y;
    const int split = blockIdx.z;
    const int nk_total = (K2 + kBK - 1) / kBK;
    const int k_begin = split * kstages_per_split;
    const int k_end = min(nk_total, k_begin + kstages_per_split);
    const int nk = max(0, k_end - k_begin);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&ready[s]), 256);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 256);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_slot;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicOr(err, code);
    };

    if (warp == 0) {
        if (lane == 0) {
            // producer
            int issued = 0;
            for (int i = 0; i < nk && !*abort_flag; ++i) {
                const int s = i % kStages;
                if (i >= kStages && !mbar_wait(smem_u32(&empty[s]), ((i / kStages) - 1) & 1, wait_ns)) {
                    fail(1);
                    break;
                }
                unsigned char* st = base + s * TB::stage;
                const unsigned fb = smem_u32(&full[s]);
                mbar_expect_tx(fb, unsigned(TB::a_raw + (PRE ? 2 : 1) * TB::b));
                const int kr = (k_begin + i) * kBK;  // real K offset
                if (OPA == 1) {
                    tma_load_2d(smem_u32(st), &mapA, kr, tile_m * (kBM / 2), fb);
                } else {
                    for (int b = 0; b < 4; ++b)
                        tma_load_2d(smem_u32(st + b * 2048), &mapA, tile_m * kBM + 32 * b, kr / 2, fb);
                }
                tma_load_2d(smem_u32(st + TB::a_raw), &mapB, kr, tile_n * BN, fb);
                if (PRE) tma_load_2d(smem_u32(st + TB::a_raw + TB::b), &mapBl, kr, tile_n * BN, fb);
                ++issued;
            }
            // drain: every load this thread issued must land before the CTA exits
            for (int i = max(0, issued - kStages); i < issued; ++i) {
                const int s = i % kStages;
                if (!mbar_wait(smem_u32(&full[s]), (i / kStages) & 1, drain_ns)) atomicOr(err, 8);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: the kAcc stages of group i / kAcc accumulate (fresh at the group's first stage) into
            // TMEM buffer (i / kAcc) & 1; A from TMEM, B from shared memory
            const unsigned idesc =
                (1u << 4) | (2u << 7) | (2u << 10) | (unsigned(BN >> 3) << 17) | (unsigned(kBM >> 4) << 24);
            int issued = 0;
            for (int i = 0; i < nk && !*abort_flag; ++i) {
                const int s = i % kStages;
                const int grp = i / kAcc;
                const int bf = grp & 1;
                const bool first = (i % kAcc) == 0;
                const bool last = (i % kAcc) == kAcc - 1 || i == nk - 1;
                if (first && grp >= 2 && !mbar_wait(smem_u32(&acc_empty[bf]), ((grp >> 1) - 1) & 1, wait_ns)) {
                    fail(32);
                    break;
                }
                if (!mbar_wait(smem_u32(&ready[s]), (i / kStages) & 1, wait_ns)) {
                    fail(2);
                    break;
                }
                tc_fence_after();
                unsigned char* st = base + s * TB::stage;
                const unsigned a_hi = tmem + a_col<BN>(s);
                const unsigned a_lo = a_hi + 32u;
                const unsigned b_hi = smem_u32(st + TB::a_raw);
                const unsigned b_lo = b_hi + TB::b;
                const unsigned d = tmem + unsigned(bf * BN);
#pragma unroll
                for (int kk = 0; kk < kBK / 8; ++kk) {
                    const unsigned long long dbh = sdesc(b_hi + kk * 32, 16, 1024, 2);
                    const unsigned long long dbl = sdesc(b_lo + kk * 32, 16, 1024, 2);
                    // small terms first, then the leading product
                    mma_tf32_ta(d, a_hi + kk * 8, dbl, idesc, (kk > 0 || !first) ? 1u : 0u);
                    mma_tf32_ta(d, a_lo + kk * 8, dbh, idesc, 1u);
                    mma_tf32_ta(d, a_hi + kk * 8, dbh, idesc, 1u);
                }
                mma_commit(smem_u32(&empty[s]));
                if (last) mma_commit(smem_u32(&acc_full[bf]));
                ++issued;
            }
            // after an abort: the MMAs issued so far complete (the commit of the last issued stage tracks all
            // of them) before TMEM is freed below
            if (*abort_flag && issued > 0) {
                const int il = issued - 1;
                if (!mbar_wait(smem_u32(&empty[il % kStages]), (il / kStages) & 1, drain_ns)) atomicOr(err, 64);
            }
        }
    } else {
        // warps 2..9: expand + split stage i's A into TMEM (and split B in shared memory unless PRE), drain
        // stage i-1, finally store.  TMEM lane quarter q = warp % 4 (the lanes this warp may access); warps
        // 2-5 handle real K [0, 16) of a stage's A and columns [0, BN/2) of C, warps 6-9 K [16, 32) and
        // columns [BN/2, BN)
        constexpr int HB = BN / 2;
        const int t = threadIdx.x - 64;  // 0..255
        const int q = warp & 3;
        const int g = (warp >= 6) ? 1 : 0;
        const int col0 = g * HB;
        const int rr = 32 * q + lane;        // real row of the tile = TMEM lane
        const int m = rr >> 1;               // complex row of op(A) within the tile
        const bool odd = (rr & 1) != 0;
        float acc[HB];
#pragma unroll
        for (int j = 0; j < HB; ++j) acc[j] = 0.f;
        bool ok = true;
        auto drain = [&](int grp) {  // the accumulator of stage group grp
            const int bf = grp & 1;
            ok = ok && mbar_wait(smem_u32(&acc_full[bf]), (grp >> 1) & 1, wait_ns);
            if (!ok) {
                fail(16);
                return;
            }
            tc_fence_after();
            const unsigned ta = tmem + (unsigned(32 * q) << 16) + unsigned(bf * BN + col0);
#pragma unroll
            for (int c0 = 0; c0 < HB; c0 += 16) {
                float v[16];
                tmem_ld16(ta + unsigned(c0), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[c0 + j] += v[j];
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&acc_empty[bf]));
        };
        for (int i = 0; i < nk && !*abort_flag; ++i) {
            const int s = i % kStages;
            if (!mbar_wait(smem_u32(&full[s]), (i / kStages) & 1, wait_ns)) {
                fail(4);
                break;
            }
            // the MMAs that last read this stage's TMEM columns have completed (they released the stage
            // before its refill landed)
            tc_fence_after();
            unsigned char* st = base + s * TB::stage;
            const unsigned char* araw = st;
            // A: this thread's real row of op(A) over its 16 real K of the stage.  Blocks of the real
            // form: "N" [[ar, -ai], [ai, ar]], "C" [[ar, ai], [-ai, ar]]; an even real row takes the first
            // row of each block, an odd one the second
            float v[16];
            if (OPA == 1) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {  // raw row m, 16-byte chunks 4g..4g+3 (two complex each)
                    const float4 x = *reinterpret_cast<const float4*>(araw + sw128(unsigned(m), unsigned(4 * g + j)));
                    v[4 * j + 0] = odd ? -x.y : x.x;
                    v[4 * j + 1] = odd ? x.x : x.y;
                    v[4 * j + 2] = odd ? -x.w : x.z;
                    v[4 * j + 3] = odd ? x.z : x.w;
                }
            } else {
                const int ml = m & 15;  // within MN block q (16 complex rows)
#pragma unroll
                for (int j = 0; j < 8; ++j) {  // raw K-rows 8g..8g+7
                    const float2 x = *reinterpret_cast<const float2*>(
                        araw + q * 2048 + sw128(unsigned(8 * g + j), unsigned(ml >> 1)) + (ml & 1) * 8);
                    v[2 * j + 0] = odd ? x.y : x.x;
                    v[2 * j + 1] = odd ? x.x : -x.y;
                }
            }
            float lo[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float h = tf32_round(v[j]);
                lo[j] = v[j] - h;
                v[j] = h;
            }
            const unsigned tal = tmem + (unsigned(32 * q) << 16) + a_col<BN>(s) + unsigned(16 * g);
            tmem_st16(tal, v);
            tmem_st16(tal + 32u, lo);
            if (!PRE) {
                // B: in-place hi, lo beside it (same layout)
                unsigned char* bhi = st + TB::a_raw;
                unsigned char* blo = bhi + TB::b;
                for (int qq = t; qq < BN * 8; qq += 256) {
                    float4* p = reinterpret_cast<float4*>(bhi + qq * 16);
                    const float4 x = *p;
                    const float4 h = make_float4(tf32_round(x.x), tf32_round(x.y), tf32_round(x.z), tf32_round(x.w));
                    *p = h;
                    *reinterpret_cast<float4*>(blo + qq * 16) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
                }
                fence_async_smem();
            }
            tmem_st_wait();
            tc_fence_before();
            mbar_arrive(smem_u32(&ready[s]));
            if (i > 0 && i % kAcc == 0) drain(i / kAcc - 1);
            if (!ok) break;
        }
        if (ok && !*abort_flag && nk > 0) drain((nk - 1) / kAcc);
        // store (warp-uniform: the shuffles are collective)
        const bool go = __all_sync(0xffffffffu, ok && !*abort_flag && nk > 0);
        if (go) {
            const int row = tile_m * kBM + rr;  // real row of C
            const bool row_ok = row < M2;
            const bool im = odd;
            const bool use_beta = (beta.x != 0.f || beta.y != 0.f);
            if (ws) {
#pragma unroll
                for (int j = 0; j < HB; ++j) {
                    const int n = tile_n * BN + col0 + j;
                    if (row_ok && n < N) ws[(size_t(split) * N + n) * size_t(M2) + row] = acc[j];
                }
            } else {
                // groups of 16 columns: all loads of C in a group are issued before any is used
                constexpr int G = 16;
#pragma unroll
                for (int j0 = 0; j0 < HB; j0 += G) {
                    float cs[G];
#pragma unroll
                    for (int j = 0; j < G; ++j) {
                        const int n = tile_n * BN + col0 + j0 + j;
                        cs[j] = (use_beta && row_ok && n < N) ? C[size_t(n) * ldc2 + row] : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < G; ++j) {
                        const int n = tile_n * BN + col0 + j0 + j;
                        const float v = acc[j0 + j];
                        const float partner = __shfl_xor_sync(0xffffffffu, v, 1);
                        // (alpha * acc): re = ar*vr - ai*vi, im = ar*vi + ai*vr
                        float out = im ? alpha.x * v + alpha.y * partner : alpha.x * v - alpha.y * partner;
                        const float cpart = __shfl_xor_sync(0xffffffffu, cs[j], 1);
                        if (use_beta) out += im ? beta.x * cs[j] + beta.y * cpart : beta.x * cs[j] - beta.y * cpart;
                        if (row_ok && n < N) C[size_t(n) * ldc2 + row] = out;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
    }
}

// B (K x N complex, pitch ldb) -> hi = tf32 rounding, lo = B - hi, both with pitch ldh (even)
__global__ void k_split_b(int K, int N, const float2* __restrict__ B, long ldb, float2* __restrict__ hi,
                          float2* __restrict__ lo, long ldh) {
    const long total = long(K) * N;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const long n = t / K, k = t - n * K;
        const float2 x = B[n * ldb + k];
        const float2 h = make_float2(tf32_round(x.x), tf32_round(x.y));
        hi[n * ldh + k] = h;
        lo[n * ldh + k] = make_float2(x.x - h.x, x.y - h.y);
    }
}

// C (+)= sum over splits, with alpha / beta, deterministic order
__global__ void k_splitk_reduce(int M2, int N, int splits, const float* __restrict__ ws, float2 alpha, float2 beta,
                                float* __restrict__ C, long ldc2) {
    const long total = long(M2 / 2) * N;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int n = int(t / (M2 / 2));
        const int a = int(t - long(n) * (M2 / 2));
        float sr = 0.f, si = 0.f;
        for (int s = 0; s < splits; ++s) {
            const float* w = ws + (size_t(s) * N + n) * size_t(M2) + 2 * a;
            sr += w[0];
            si += w[1];
        }
        float* cp = C + size_t(n) * ldc2 + 2 * a;
        float orr = alpha.x * sr - alpha.y * si, oi = alpha.x * si + alpha.y * sr;
        if (beta.x != 0.f || beta.y != 0.f) {
            const float cr = cp[0], ci = cp[1];
            orr += beta.x * cr - beta.y * ci;
            oi += beta.x * ci + beta.y * cr;
        }
        cp[0] = orr;
        cp[1] = oi;
    }
}

// 2-D fp32 tensor map: inner extent `inner` floats, `outer` rows of pitch `pitch_floats`
CUtensorMap make_map(const void* base, long inner, long outer, long pitch_floats, unsigned box_inner, unsigned box_outer) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {cuuint64_t(inner), cuuint64_t(outer)};
    const cuuint64_t strides[1] = {cuuint64_t(pitch_floats) * 4};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box,
                                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    B200_CHECK(r == CUDA_SUCCESS, kInvalidArgument, "cuTensorMapEncodeTiled failed (code " + std::to_string(int(r)) + ")");
    return m;
}

std::atomic<unsigned long long> g_wait_ns{kWaitNs};
unsigned long long wait_limit_ns() { return g_wait_ns.load(std::memory_order_relaxed); }

template <int BN, int OPA, int PRE> void set_attr_once() {
    static std::once_flag once;
    std::call_once(once, [] {
        B200_CUDA(cudaFuncSetAttribute(k_tc_cgemm<BN, OPA, PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TileBytes<BN>::total));
    });
}

template <int BN, int OPA>
void launch(int M, int N, int K, float2 alpha, const float2* A, int lda, const float2* B, int ldb, float2 beta, float2* C,
            int ldc, TcGemmWorkspace& w, cudaStream_t s) {
    const int M2 = 2 * M, K2 = 2 * K;
    CUtensorMap mA = (OPA == 1) ? make_map(A, 2L * K, M, 2L * lda, 32, 64)   // rows of A^H = columns of A
                                : make_map(A, 2L * M, K, 2L * lda, 32, 16);  // columns of A, MN-major
    const int tm = (M2 + kBM - 1) / kBM, tn = (N + BN - 1) / BN;
    // when many M tiles read B (tall op(A): the H|psi> and subspace updates), B is split into hi / lo once
    // here and the CTAs only copy it; otherwise every CTA splits its B tiles in shared memory
    const bool pre = tm >= 16;
    CUtensorMap mB, mBl;
    if (pre) {
        const long ldh = long(K) + (K & 1);  // even: 16-byte row pitch
        w.bsplit.resize(size_t(2) * size_t(ldh) * N);
        float2* hi = w.bsplit.ptr;
        float2* lo = hi + size_t(ldh) * N;
        const long total = long(K) * N;
        int blocks = int((total + 255) / 256);
        if (blocks > 148 * 8) blocks = 148 * 8;
        k_split_b<<<blocks, 256, 0, s>>>(K, N, B, ldb, hi, lo, ldh);
        note_launch();
        B200_CUDA(cudaGetLastError());
        mB = make_map(hi, 2L * K, N, 2L * ldh, 32, BN);
        mBl = make_map(lo, 2L * K, N, 2L * ldh, 32, BN);
    } else {
        mB = make_map(B, 2L * K, N, 2L * ldb, 32, BN);
        mBl = mB;
    }
    const int nk = (K2 + kBK - 1) / kBK;
    // split K so that whole waves of one CTA per SM (148 SMs) are filled.  Cost in microseconds:
    // waves * stages-per-CTA at about 1 us per CTA stage, plus for sp > 1 the reduction's traffic
    // (the partial sums written by the GEMM and read back, C read and written: (2 sp + 2) * M * N * 8
    // bytes at about 6 TB/s) and its launch
    int splits = 1;
    {
        const long tiles = long(tm) * tn;
        const double mn_us = double(M) * double(N) * 8.0 / 6.0e6;
        double best = 1e300;
        const int smax = nk < 1024 ? nk : 1024;
        for (int sp = 1; sp <= smax; ++sp) {
            if (sp > 1 && w.ws_cap && size_t(sp) * size_t(N) * size_t(M2) > w.ws_cap) break;
            const long per_s = (nk + sp - 1) / sp;
            const long waves = (tiles * sp + 147) / 148;
            const double cost = double(waves) * double(per_s) + (sp > 1 ? (2.0 * sp + 2.0) * mn_us + 4.0 : 0.0);
            if (cost < best - 1e-9) {
                best = cost;
                splits = sp;
            }
        }
    }
    const int per = (nk + splits - 1) / splits;
    splits = (nk + per - 1) / per;
    float* ws = nullptr;
    if (splits > 1) {
        w.ws.resize(size_t(splits) * N * M2);
        ws = w.ws.ptr;
    }
    B200_CHECK((OPA == 0 ? tm : tn) <= 65535, kInvalidArgument, "tc_cgemm: too many tiles for the grid");
    const dim3 grid = OPA == 0 ? dim3(tn, tm, splits) : dim3(tm, tn, splits);
    if (pre) {
        set_attr_once<BN, OPA, 1>();
        k_tc_cgemm<BN, OPA, 1><<<grid, kThreads, TileBytes<BN>::total, s>>>(
            mA, mB, mBl, M2, N, K2, per, alpha, beta, reinterpret_cast<float*>(C), 2L * ldc, ws, w.err.ptr, wait_limit_ns());
    } else {
        set_attr_once<BN, OPA, 0>();
        k_tc_cgemm<BN, OPA, 0><<<grid, kThreads, TileBytes<BN>::total, s>>>(
            mA, mB, mBl, M2, N, K2, per, alpha, beta, reinterpret_cast<float*>(C), 2L * ldc, ws, w.err.ptr, wait_limit_ns());
    }
    note_launch();
    B200_CUDA(cudaGetLastError());
    if (splits > 1) {
        const long total = long(M) * N;
        int blocks = int((total + 255) / 256);
        if (blocks > 148 * 8) blocks = 148 * 8;
        k_splitk_reduce<<<blocks, 256, 0, s>>>(M2, N, splits, ws, alpha, beta, reinterpret_cast<float*>(C), 2L * ldc);
        note_launch();
        B200_CUDA(cudaGetLastError());
    }
}

}  // namespace

void TcGemmWorkspace::ensure() {
    if (!err.ptr) {
        err.resize(1);
        B200_CUDA(cudaMemset(err.ptr, 0, sizeof(int)));
    }
}

void TcGemmWorkspace::reserve(size_t ws_floats, size_t bsplit_elems) {
    ensure();
    ws_cap = ws_floats;
    ws.resize(ws_floats);
    bsplit.resize(bsplit_elems);
}

int TcGemmWorkspace::read_error(cudaStream_t s) {
    int h = 0;
    if (err.ptr) {
        B200_CUDA(cudaMemcpyAsync(&h, err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
        B200_CUDA(cudaStreamSynchronize(s));
        if (h) B200_CUDA(cudaMemsetAsync(err.ptr, 0, sizeof(int), s));  // reported once, then cleared
    }
    return h;
}

void set_tc_wait_limit_ns(unsigned long long ns) { g_wait_ns.store(ns ? ns : kWaitNs, std::memory_order_relaxed); }
unsigned long long tc_wait_limit_ns() { return wait_limit_ns(); }

void tc_cgemm(char opa, int M, int N, int K, float2 alpha, const float2* A, int lda, const float2* B, int ldb,
              float2 beta, float2* C, int ldc, TcGemmWorkspace& w, cudaStream_t s) {
    B200_CHECK(opa == 'N' || opa == 'C', kInvalidArgument, "tc_cgemm: op(A) must be 'N' or 'C'");
    B200_CHECK(M > 0 && N > 0 && K > 0, kInvalidArgument, "tc_cgemm: empty problem");
    B200_CHECK(lda % 2 == 0 && ldb % 2 == 0, kInvalidArgument,
               "tc_cgemm: lda and ldb must be even (16-byte row pitch for TMA)");
    B200_CHECK(ldc >= M, kInvalidArgument, "tc_cgemm: ldc < M");
    B200_CHECK((reinterpret_cast<uintptr_t>(A) & 15) == 0 && (reinterpret_cast<uintptr_t>(B) & 15) == 0, kInvalidArgument,
               "tc_cgemm: A and B must be 16-byte aligned");
    B200_CHECK(opa == 'C' ? lda >= K : lda >= M, kInvalidArgument, "tc_cgemm: lda too small");
    B200_CHECK(ldb >= K, kInvalidArgument, "tc_cgemm: ldb < K");
    w.ensure();
    if (N <= 64) {
        if (opa == 'N') launch<64, 0>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, w, s);
        else launch<64, 1>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, w, s);
    } else {
        if (opa == 'N') launch<128, 0>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, w, s);
        else launch<128, 1>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, w, s);
    }
}

}  // namespace b200
