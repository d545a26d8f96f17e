// FP64 complex GEMM on the int8 tensor cores: exact modular (Chinese-remainder) emulation.
//
// Real form.  C = op(A) B with complex entries is two real products over K' = 2K interleaved reals: a row
// of op(A) becomes A' = [ar_0, ai_0, ar_1, ai_1, ...] (the raw entries of the row of A for op 'N', of the
// column of A for op 'C'), and a complex column of B becomes two real rows of B':
//   op 'N':  re = [br, -bi, ...],  im = [bi, br, ...]      (C = A B)
//   op 'C':  re = [br,  bi, ...],  im = [bi, -br, ...]     (C = A^H B)
// so that C_re = A' . B'_re and C_im = A' . B'_im: one real GEMM of M x 2N x 2K.
//
// Integers.  Each row of A' is multiplied by 2^e (e per row) so that its largest magnitude is below 2^q and
// rounded to integers; the same for the rows of B' (one exponent per complex column).  With M = prod m_l
// over n pairwise coprime moduli m_l <= 256 and 2q + log2 K' + 2 <= log2 M, the integer product satisfies
// |C'| <= K' 2^2q <= M / 4, so C' is fixed by its residues mod every m_l.  For n = 16 (log2 M = 125.4) and
// K' <= 2^18, q >= 52: the largest entry of every row keeps all its bits.  The exponents come from maxima,
// which neither overflow nor underflow and do not depend on the order of a reduction.
//
// Per modulus.  Residues of the integers in the symmetric range (|r| <= 128, int8), K-major, one plane per
// modulus; one int8 GEMM per modulus on tcgen05 (kind::i8, int32 accumulation in tensor memory, exact while
// K' per split <= 130944: 128 * 128 * 130944 < 2^31); the epilogue keeps the product mod m_l (one byte).
//
// Recombination.  C' = sum_l c_l w_l  (mod M), w_l = (M / m_l) ((M / m_l)^-1 mod m_l).  In units of M:
// C' / M = frac(sum_l c_l u_l) with u_l = w_l / M = wa_l + wb_l, wa_l holding the first 40 fraction bits:
// sum_l c_l wa_l is exact in FP64 (c_l < 2^8, at most 16 terms, 40 fraction bits: 52 bits), and
// sum_l c_l wb_l < 2^-32 carries rounding errors near 2^-82.  x = frac in [-1/2, 1/2) is rounded once,
// relative to itself, when the small sum is added; C' = x M and C = C' 2^-(e_row + e_col).  So C' is
// accurate to a few ulps of itself plus about 2^-80 of its bound M / 4, and the error of C is that of
// rounding op(A) and B to q-bit integers (half a unit of 2^-q of each row's largest entry).
//
// Kernels: row / column maxima (per segment), residues (8 bytes per modulus per store),
// the tcgen05 GEMM of all moduli and K splits in one launch, and the recombination (alpha, beta).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "gemm_oz.h"
#include "gemm_tc.h"
#include "tcgen05_util.cuh"

namespace b200 {
namespace {

using namespace tcu;

// pairwise coprime; the first modulus is 256 (oz_res relies on it)
constexpr int kOzMods[kOzMaxMods] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};
constexpr int kOzNonFinite = -2147483647 - 1;  // row exponent marking a row with a NaN or infinite entry
constexpr int kOzSeg = 4096;                   // complex entries per column segment of the norm / residue kernels
constexpr int kOzMaxKbPerSplit = 1023;         // 128-byte K blocks per split: 1023 * 128 = 130944 reals
constexpr int kOzThreads = 320;                // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr int kOzATile = 128 * 128;            // bytes of one A stage: 128 rows x 128 K
constexpr int kOzSmem = 227 * 1024;            // dynamic shared memory per CTA: one persistent CTA per SM

struct OzConst {
    int n, q;  // q: set per call from K' (oz_scale_bits)
    unsigned m[kOzMaxMods], magic[kOzMaxMods];             // magic = ceil(2^32 / m)
    unsigned c21[kOzMaxMods], c42[kOzMaxMods], off62[kOzMaxMods], c31[kOzMaxMods];
    unsigned h[kOzMaxMods];  // residues are kept shifted by h: 128 for m = 256, (m - 1) / 2 for odd m
    double wa[kOzMaxMods], wb[kOzMaxMods];
    double mprod, log2m;
};

using u128 = unsigned __int128;
double u128_to_double(u128 x) {
    return std::ldexp(double((unsigned long long)(x >> 64)), 64) + double((unsigned long long)x);
}

OzConst make_const(int n) {
    OzConst c{};
    c.n = n;
    u128 M = 1;
    double log2m = 0.0;
    for (int l = 0; l < n; ++l) {
        M *= u128(kOzMods[l]);
        log2m += std::log2(double(kOzMods[l]));
    }
    c.q = 0;
    c.log2m = log2m;
    for (int l = 0; l < n; ++l) {
        const unsigned m = unsigned(kOzMods[l]);
        c.m[l] = m;
        c.magic[l] = unsigned(((1ull << 32) + m - 1) / m);
        c.c21[l] = unsigned((1ull << 21) % m);
        c.c42[l] = unsigned((1ull << 42) % m);
        c.h[l] = m == 256 ? 128u : (m - 1) / 2;
        c.off62[l] = unsigned((m - (1ull << 62) % m + c.h[l]) % m);
        c.c31[l] = unsigned((1ull << 31) % m);
        const u128 Ml = M / m;
        const unsigned r = unsigned(Ml % m);
        unsigned y = 1;
        while ((u128(r) * y) % m != 1) ++y;  // the inverse of M / m_l mod m_l (m_l <= 256)
        const u128 w = (Ml * y) % M;         // Ml < 2^118, y < 2^8: no overflow
        u128 rem = w;
        unsigned long long a = 0;
        for (int b = 0; b < 40; ++b) {  // the first 40 bits of w / M (2 rem < 2M < 2^127)
            rem <<= 1;
            a <<= 1;
            if (rem >= M) {
                rem -= M;
                a |= 1;
            }
        }
        c.wa[l] = std::ldexp(double(a), -40);
        c.wb[l] = std::ldexp(u128_to_double(rem) / u128_to_double(M), -40);
    }
    c.mprod = u128_to_double(M);
    return c;
}

const OzConst& oz_const_table(int n) {
    static OzConst table[kOzMaxMods - kOzMinMods + 1];
    static std::once_flag once;
    std::call_once(once, [] {
        for (int k = kOzMinMods; k <= kOzMaxMods; ++k) table[k - kOzMinMods] = make_const(k);
    });
    B200_CHECK(n >= kOzMinMods && n <= kOzMaxMods, kInvalidArgument, "int8 GEMM: number of moduli must be 12..16");
    return table[n - kOzMinMods];
}
// the constants of n moduli with q for real rows of length kr: 2q + log2(kr) + 2 <= log2 M
OzConst oz_const(int n, long kr) {
    OzConst c = oz_const_table(n);
    c.q = int(std::floor((c.log2m - 2.0 - std::log2(double(kr > 1 ? kr : 1))) / 2.0));
    B200_CHECK(c.q >= 30 && c.q <= 61, kInvalidArgument, "int8 GEMM: K too long for the number of moduli");
    return c;
}

// x mod m for x < 2^32 (q = floor(x / m) or one more)
__device__ __forceinline__ unsigned oz_umod(unsigned x, unsigned m, unsigned magic) {
    const unsigned q = __umulhi(x, magic);
    const int r = int(x - q * m);
    return unsigned(r < 0 ? r + int(m) : r);
}
// (u - 2^62 + h) mod m for u < 2^63: three 21-bit pieces
__device__ __forceinline__ unsigned oz_res(unsigned long long u, const OzConst& c, int l) {
    if (l == 0) return (unsigned(u) + 128u) & 0xFFu;  // m_0 = 256 (h = 128): 2^62 = 0 mod 256
    const unsigned p0 = unsigned(u) & 0x1FFFFFu, p1 = unsigned(u >> 21) & 0x1FFFFFu, p2 = unsigned(u >> 42);
    return oz_umod(p2 * c.c42[l] + p1 * c.c21[l] + p0 + c.off62[l], c.m[l], c.magic[l]);
}
// x 2^e rounded to the nearest integer, offset by 2^62 (|x| 2^e < 2^62): two exact scalings by powers of two
// (2^e itself may lie outside the double range), then one rounding conversion
__device__ __forceinline__ double oz_pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }
struct OzScale {
    double s1, s2;
    __device__ explicit OzScale(int e) {
        const int e1 = e < 1000 ? e : 1000;  // e >= q - 1024 > -1022: both factors are normal doubles
        s1 = oz_pow2(e1);
        s2 = oz_pow2(e - e1);
    }
    __device__ unsigned long long operator()(double x) const {
        return (unsigned long long)(__double2ll_rn((x * s1) * s2) + (1ll << 62));
    }
};
// the symmetric representative (as a byte) of v, and of -v, from r = (v + h) mod m: r - h lies in
// [-128, 127] for m = 256 and in [-(m-1)/2, (m-1)/2] for odd m; h - r is -v's (128 = -128 as a byte, m = 256)
__device__ __forceinline__ unsigned oz_sym(unsigned r, unsigned h) { return (r - h) & 0xFFu; }
__device__ __forceinline__ unsigned oz_symneg(unsigned r, unsigned h) { return (h - r) & 0xFFu; }

// exponent e of a row whose largest magnitude is mx: mx 2^e < 2^q (kOzNonFinite for NaN / infinity)
__device__ __forceinline__ int oz_exponent(double mx, int q) {
    if (!(mx <= 1.7976931348623157e308)) return kOzNonFinite;
    if (mx == 0.0) return 0;
    int E;
    frexp(mx, &E);  // mx = f 2^E, f in [0.5, 1)
    return q - E;
}
// largest magnitude of the real and imaginary parts seen so far; a NaN or infinity turns it into +inf
__device__ __forceinline__ double oz_amax(double m, double2 x) {
    const double a = fabs(x.x), b = fabs(x.y);
    if (!(a <= 1.7976931348623157e308) || !(b <= 1.7976931348623157e308)) return __longlong_as_double(0x7ff0000000000000ll);
    return fmax(m, fmax(a, b));
}

__device__ __forceinline__ double block_max256(double v) {
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < 8; ++w) s = fmax(s, red[w]);
    return s;
}

// largest magnitude over segment blockIdx.x of column blockIdx.y (K complex entries, pitch ld) -> part[col][seg]
__global__ void __launch_bounds__(256) k_oz_absmax_cols(int K, const double2* __restrict__ X, long ld,
                                                        double* __restrict__ part) {
    const int j = blockIdx.y, sg = blockIdx.x;
    const long k0 = long(sg) * kOzSeg, k1 = min(long(K), k0 + kOzSeg);
    const double2* col = X + long(j) * ld;
    double m = 0.0;
    for (long k = k0 + threadIdx.x; k < k1; k += 256) m = oz_amax(m, col[k]);
    m = block_max256(m);
    if (threadIdx.x == 0) part[long(j) * gridDim.x + sg] = m;
}

// residues of columns (segment blockIdx.x of column j = blockIdx.y; 4 complex entries per thread step).
// KIND 0: one real row per column, [re, im] (op(A) rows for op 'C').  KIND 1 / 2: two real rows per column,
// the B' rows of op 'N' / op 'C'.  exps[j]: the column's exponent.
template <int KIND>
__global__ void __launch_bounds__(256) k_oz_res_cols(int K, const double2* __restrict__ X, long ld,
                                                     const double* __restrict__ part, const __grid_constant__ OzConst c,
                                                     signed char* __restrict__ res, long kp, long plane,
                                                     int* __restrict__ exps) {
    const int j = blockIdx.y, sg = blockIdx.x, nseg = gridDim.x;
    __shared__ int s_e;
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int t = 0; t < nseg; ++t) mx = fmax(mx, part[long(j) * nseg + t]);
        const int e = oz_exponent(mx, c.q);
        s_e = e;
        if (sg == 0) exps[j] = e;
    }
    __syncthreads();
    const int e = s_e;
    const bool bad = e == kOzNonFinite;
    const double2* col = X + long(j) * ld;
    const long k0 = long(sg) * kOzSeg, k1 = min(long(K), k0 + kOzSeg);
    const OzScale scale(bad ? 0 : e);
    for (long kb = k0 + 4L * threadIdx.x; kb < k1; kb += 4L * 256) {
        unsigned long long ur[4], ui[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const long k = kb + t;
            const double2 x = (k < k1 && !bad) ? col[k] : make_double2(0.0, 0.0);
            ur[t] = scale(x.x);
            ui[t] = scale(x.y);
        }
#pragma unroll
        for (int l = 0; l < kOzMaxMods; ++l) {
            if (l >= c.n) break;
            const unsigned hs = c.h[l];
            unsigned rr[4], ri[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                rr[t] = oz_res(ur[t], c, l);
                ri[t] = oz_res(ui[t], c, l);
            }
            signed char* pl = res + long(l) * plane + 2 * kb;
            if (KIND == 0) {
                uint2 v;
                v.x = oz_sym(rr[0], hs) | (oz_sym(ri[0], hs) << 8) | (oz_sym(rr[1], hs) << 16) | (oz_sym(ri[1], hs) << 24);
                v.y = oz_sym(rr[2], hs) | (oz_sym(ri[2], hs) << 8) | (oz_sym(rr[3], hs) << 16) | (oz_sym(ri[3], hs) << 24);
                *reinterpret_cast<uint2*>(pl + long(j) * kp) = v;
            } else {
                uint2 vre, vim;
                if (KIND == 1) {  // re = [br, -bi], im = [bi, br]
                    vre.x = oz_sym(rr[0], hs) | (oz_symneg(ri[0], hs) << 8) | (oz_sym(rr[1], hs) << 16) | (oz_symneg(ri[1], hs) << 24);
                    vre.y = oz_sym(rr[2], hs) | (oz_symneg(ri[2], hs) << 8) | (oz_sym(rr[3], hs) << 16) | (oz_symneg(ri[3], hs) << 24);
                    vim.x = oz_sym(ri[0], hs) | (oz_sym(rr[0], hs) << 8) | (oz_sym(ri[1], hs) << 16) | (oz_sym(rr[1], hs) << 24);
                    vim.y = oz_sym(ri[2], hs) | (oz_sym(rr[2], hs) << 8) | (oz_sym(ri[3], hs) << 16) | (oz_sym(rr[3], hs) << 24);
                } else {  // re = [br, bi], im = [bi, -br]
                    vre.x = oz_sym(rr[0], hs) | (oz_sym(ri[0], hs) << 8) | (oz_sym(rr[1], hs) << 16) | (oz_sym(ri[1], hs) << 24);
                    vre.y = oz_sym(rr[2], hs) | (oz_sym(ri[2], hs) << 8) | (oz_sym(rr[3], hs) << 16) | (oz_sym(ri[3], hs) << 24);
                    vim.x = oz_sym(ri[0], hs) | (oz_symneg(rr[0], hs) << 8) | (oz_sym(ri[1], hs) << 16) | (oz_symneg(rr[1], hs) << 24);
                    vim.y = oz_sym(ri[2], hs) | (oz_symneg(rr[2], hs) << 8) | (oz_sym(ri[3], hs) << 16) | (oz_symneg(rr[3], hs) << 24);
                }
                *reinterpret_cast<uint2*>(pl + long(2 * j) * kp) = vre;
                *reinterpret_cast<uint2*>(pl + long(2 * j + 1) * kp) = vim;
            }
        }
    }
}

// largest magnitude over row r of a column-major M x K matrix (one thread per row; coalesced along rows)
__global__ void k_oz_absmax_rows(int M, int K, const double2* __restrict__ X, long ld, double* __restrict__ part) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M) return;
    double m = 0.0;
    for (int k = 0; k < K; ++k) m = oz_amax(m, X[r + long(k) * ld]);
    part[r] = m;
}

// residues of the rows of a column-major M x K matrix: a 32-row x 32-column tile per block (32 x 8 threads),
// loaded along rows and written along K through shared memory
__global__ void __launch_bounds__(256) k_oz_res_rows(int M, int K, const double2* __restrict__ X, long ld,
                                                     const double* __restrict__ part, const __grid_constant__ OzConst c,
                                                     signed char* __restrict__ res, long kp, long plane,
                                                     int* __restrict__ exps) {
    __shared__ __align__(16) unsigned char tile[kOzMaxMods][32][72];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    const int row = r0 + tx;
    const int e = row < M ? oz_exponent(part[row], c.q) : 0;
    if (blockIdx.x == 0 && ty == 0 && row < M) exps[row] = e;
    const bool bad = e == kOzNonFinite;
    const OzScale scale(bad ? 0 : e);
    for (int kk = ty; kk < 32; kk += 8) {
        const int k = k0 + kk;
        const double2 x = (row < M && k < K && !bad) ? X[row + long(k) * ld] : make_double2(0.0, 0.0);
        const unsigned long long ur = scale(x.x), ui = scale(x.y);
#pragma unroll
        for (int l = 0; l < kOzMaxMods; ++l) {
            if (l >= c.n) break;
            tile[l][tx][2 * kk] = (unsigned char)oz_sym(oz_res(ur, c, l), c.h[l]);
            tile[l][tx][2 * kk + 1] = (unsigned char)oz_sym(oz_res(ui, c, l), c.h[l]);
        }
    }
    __syncthreads();
    const int t = ty * 32 + tx;
    for (int qq = t; qq < c.n * 256; qq += 256) {
        const int l = qq >> 8, rr = (qq >> 3) & 31, ch = qq & 7;
        const int r = r0 + rr;
        const long off = 2L * k0 + 8L * ch;
        if (r < M && off < kp)
            *reinterpret_cast<uint2*>(res + long(l) * plane + long(r) * kp + off) =
                *reinterpret_cast<const uint2*>(&tile[l][rr][8 * ch]);
    }
}

// D (TMEM, int32) (+)= A (shared-memory descriptor, int8) * B (shared-memory descriptor, int8)
__device__ __forceinline__ void mma_i8(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                       unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tmem_ld16i(unsigned taddr, int* v) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = int(r[i]);
}

// 32 consecutive TMEM columns of this thread's lane in one load (one wait for all of them)
__device__ __forceinline__ void tmem_ld32i(unsigned taddr, int* v) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = int(r[i]);
}

struct OzMods {
    unsigned m[kOzMaxMods], magic[kOzMaxMods], c31[kOzMaxMods];
};

// The work of one GEMM launch: tiles of 128 msub rows (op(A)) x BN real columns (B') for every plane
// z = split * n + l (modulus l, K split `split`).  Streaming schedule: tile t = blockIdx.x + i gridDim.x with
// tile_n fastest, then tile_m, then z (the CTAs running together share their A and B tiles through L2).
// Resident schedule (B' of one (z, tile_n) fits in shared memory): a fixed tile_n and a contiguous range of
// (z, tile_m) per CTA, z major, so that a CTA loads B' once per plane z it meets.
struct OzSched {
    int tm, tn, nz, per_split, nk_total, msub, nbuf;
    bool resident;
};
struct OzTile {
    int tile_m, tile_n, z, pair, k_begin, nk;
};
struct OzIter {
    long t, t_end, step;
    int tile_n;  // resident schedule: this CTA's column tile
    __device__ explicit OzIter(const OzSched& s) {
        const long T = long(s.tm) * s.tn * s.nz;
        if (s.resident) {
            // CTA c takes column tile c % tn and chunk c / tn of the (z, tile_m) sequence: the tn CTAs of a
            // group walk the same A tiles at the same pace, so A crosses HBM once
            const long U = long(s.tm) * s.nz;
            const int groups = gridDim.x / s.tn;
            const int grp = blockIdx.x / s.tn;
            tile_n = blockIdx.x % s.tn;
            const long chunk = (U + groups - 1) / groups;
            t = grp < groups ? long(grp) * chunk : U;
            t_end = min(U, t + chunk);
            step = 1;
        } else {
            t = blockIdx.x;
            t_end = T;
            step = gridDim.x;
        }
    }
    // the next tile of this CTA with its K range (n moduli per split)
    __device__ bool next(const OzSched& s, int n, OzTile& o) {
        if (t >= t_end) return false;
        if (s.resident) {
            o.z = int(t / s.tm);
            o.tile_m = int(t % s.tm);
            o.tile_n = tile_n;
            o.pair = o.z * s.tn + tile_n;
        } else {
            o.tile_n = int(t % s.tn);
            const long r = t / s.tn;
            o.tile_m = int(r % s.tm);
            o.z = int(r / s.tm);
            o.pair = o.z * s.tn + o.tile_n;
        }
        o.k_begin = (o.z / n) * s.per_split;
        o.nk = max(0, min(s.nk_total, o.k_begin + s.per_split) - o.k_begin);
        t += step;
        return true;
    }
};

constexpr int kOzEpiWarps = 8;  // warps 2..9: two per tensor-memory lane quarter

// Persistent CTAs (one per SM): warp 0 issues the TMA loads, warp 1 allocates tensor memory and issues the
// MMAs into msub accumulators of BN int32 columns per tile (two such sets 256 columns apart when they fit:
// the next tile accumulates while the last one drains), warps 2-9 drain: residues of the products mod m_l,
// stored 16 columns per thread and store in column groups, prod[((z * cgroups + cg) * rows_pad + row) * 16 + i]
// (column 16 cg + i), so that both the stores here and the loads of the recombination are coalesced.
// Every wait is bounded; a wait that runs out sets err and the CTA drains its copies and MMAs in flight and
// returns.
__global__ void __launch_bounds__(kOzThreads, 1)
    k_oz_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int rowsA, int BN,
              int stages, int n, const OzSched sc, const __grid_constant__ OzMods md, unsigned char* __restrict__ prod,
              long rows_pad, int cgroups, int* __restrict__ err, unsigned long long wait_ns) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const unsigned long long drain_ns = wait_ns > kWaitNs ? wait_ns : kWaitNs;
    unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int a_stage = sc.msub * kOzATile;
    const int b_box = BN * 128;  // one B' box: BN rows x 128 K bytes
    const int a_area = stages * a_stage;
    const int b_area = sc.resident ? sc.per_split * b_box : stages * b_box;
    unsigned char* a_st = base;
    unsigned char* b_st = base + a_area;
    unsigned long long* full = reinterpret_cast<unsigned long long*>(base + a_area + b_area);
    unsigned long long* empty = full + stages;
    unsigned long long* acc_full = empty + stages;  // [2]
    unsigned long long* acc_empty = acc_full + 2;   // [2]
    unsigned long long* bfull = acc_empty + 2;
    unsigned long long* bempty = bfull + 1;
    unsigned long long* drain = bempty + 1;
    unsigned* tmem_slot = reinterpret_cast<unsigned*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nbuf = sc.nbuf;

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 32 * kOzEpiWarps);
        }
        mbar_init(smem_u32(bfull), 1);
        mbar_init(smem_u32(bempty), 1);
        mbar_init(smem_u32(drain), 1);
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
            long g = 0;  // A stages issued (all tiles)
            int bp = 0, cur_pair = -1;
            OzIter it(sc);
            OzTile o;
            bool ok = true;
            while (ok && !*abort_flag && it.next(sc, n, o)) {
                const int l = o.z % n;
                if (sc.resident && o.pair != cur_pair) {
                    // the MMAs that read the previous B' have completed before it is overwritten
                    if (bp > 0 && !mbar_wait(smem_u32(bempty), (bp - 1) & 1, wait_ns)) {
                        fail(1);
                        break;
                    }
                    mbar_expect_tx(smem_u32(bfull), unsigned(o.nk * b_box));
                    for (int kb = 0; kb < o.nk; ++kb)
                        tma_load_3d(smem_u32(b_st + kb * b_box), &mapB, (o.k_begin + kb) * 128, o.tile_n * BN, l,
                                    smem_u32(bfull));
                    ++bp;
                    cur_pair = o.pair;
                }
                for (int i = 0; i < o.nk; ++i, ++g) {
                    const int s = int(g % stages);
                    if (g >= stages && !mbar_wait(smem_u32(&empty[s]), unsigned((g / stages) - 1) & 1u, wait_ns)) {
                        fail(1);
                        ok = false;
                        break;
                    }
                    const unsigned fb = smem_u32(&full[s]);
                    mbar_expect_tx(fb, unsigned(a_stage + (sc.resident ? 0 : b_box)));
                    const int kx = (o.k_begin + i) * 128;
                    for (int u = 0; u < sc.msub; ++u)
                        tma_load_3d(smem_u32(a_st + s * a_stage + u * kOzATile), &mapA, kx,
                                    (o.tile_m * sc.msub + u) * 128, l, fb);
                    if (!sc.resident) tma_load_3d(smem_u32(b_st + s * b_box), &mapB, kx, o.tile_n * BN, l, fb);
                }
            }
            // every copy this thread issued lands before the CTA exits
            for (long i = g - stages > 0 ? g - stages : 0; i < g; ++i)
                if (!mbar_wait(smem_u32(&full[i % stages]), unsigned(i / stages) & 1u, drain_ns)) atomicOr(err, 8);
            if (bp > 0 && !mbar_wait(smem_u32(bfull), (bp - 1) & 1, drain_ns)) atomicOr(err, 8);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // D = S32, A and B signed 8-bit, both K-major, N = BN, M = 128
            const unsigned idesc = (2u << 4) | (1u << 7) | (1u << 10) | (unsigned(BN >> 3) << 17) | (8u << 24);
            long g = 0;
            int j = 0, bp = 0, cur_pair = -1, issued = 0;
            OzIter it(sc);
            OzTile o;
            bool ok = true;
            while (ok && !*abort_flag && it.next(sc, n, o)) {
                const int b = j % nbuf;
                if (j >= nbuf && !mbar_wait(smem_u32(&acc_empty[b]), unsigned((j / nbuf) - 1) & 1u, wait_ns)) {
                    fail(32);
                    break;
                }
                if (sc.resident && o.pair != cur_pair) {
                    if (bp > 0) mma_commit(smem_u32(bempty));  // completes with every MMA on the previous B'
                    if (!mbar_wait(smem_u32(bfull), bp & 1, wait_ns)) {
                        fail(2);
                        break;
                    }
                    ++bp;
                    cur_pair = o.pair;
                }
                tc_fence_after();
                const unsigned d0 = tmem + unsigned(b * 256);
                for (int i = 0; i < o.nk; ++i, ++g) {
                    const int s = int(g % stages);
                    if (!mbar_wait(smem_u32(&full[s]), unsigned(g / stages) & 1u, wait_ns)) {
                        fail(2);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const unsigned bs = smem_u32(b_st + (sc.resident ? i : s) * b_box);
                    for (int u = 0; u < sc.msub; ++u) {
                        const unsigned a = smem_u32(a_st + s * a_stage + u * kOzATile);
                        const unsigned d = d0 + unsigned(u * BN);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            mma_i8(d, sdesc(a + kk * 32, 16, 1024, 2), sdesc(bs + kk * 32, 16, 1024, 2), idesc,
                                   (i > 0 || kk > 0) ? 1u : 0u);
                    }
                    mma_commit(smem_u32(&empty[s]));
                    ++issued;
                }
                if (!ok) break;
                if (o.nk > 0) mma_commit(smem_u32(&acc_full[b]));
                else mbar_arrive(smem_u32(&acc_full[b]));
                ++j;
            }
            // after an abort: every MMA issued so far completes before tensor memory is freed
            if (*abort_flag && issued > 0) {
                mma_commit(smem_u32(drain));
                if (!mbar_wait(smem_u32(drain), 0, drain_ns)) atomicOr(err, 64);
            }
        }
    } else {
        const int q = warp & 3;          // lane quarter this warp may access
        const int grp = (warp - 2) >> 2;  // 0: warps 2-5, 1: warps 6-9 (alternate 16-column chunks)
        const int rl = 32 * q + lane;
        int j = 0;
        OzIter it(sc);
        OzTile o;
        while (!*abort_flag && it.next(sc, n, o)) {
            const int b = j % nbuf;
            bool ok = mbar_wait(smem_u32(&acc_full[b]), unsigned(j / nbuf) & 1u, wait_ns);
            if (!ok) fail(16);
            ok = __all_sync(0xffffffffu, ok && !*abort_flag);
            if (!ok) break;
            tc_fence_after();
            const int l = o.z % n;
            const unsigned m = md.m[l], magic = md.magic[l], c31 = md.c31[l];
            for (int u = 0; u < sc.msub; ++u) {
                const int row = (o.tile_m * sc.msub + u) * 128 + rl;
                // chunks of 32 columns (16 at the tail) dealt to the two warp groups in turn: one TMEM load
                // and one wait per chunk
                for (int c0 = 32 * grp; c0 < BN; c0 += 64) {
                    const int w32 = BN - c0 >= 32 ? 32 : 16;
                    int v[32];
                    const unsigned ta = tmem + (unsigned(32 * q) << 16) + unsigned(b * 256 + u * BN + c0);
                    if (o.nk == 0) {
#pragma unroll
                        for (int t = 0; t < 32; ++t) v[t] = 0;
                    } else if (w32 == 32) {
                        tmem_ld32i(ta, v);
                    } else {
                        tmem_ld16i(ta, v);
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        if (h * 16 >= w32) break;
                        unsigned w[4];
#pragma unroll
                        for (int t4 = 0; t4 < 4; ++t4) {
                            unsigned word = 0;
#pragma unroll
                            for (int t = 0; t < 4; ++t) {
                                // (v + 2^31) mod m, then minus 2^31 mod m
                                const unsigned r = oz_umod(unsigned(v[16 * h + 4 * t4 + t]) + 0x80000000u, m, magic);
                                const int x = int(r) - int(c31);
                                word |= unsigned(x < 0 ? x + int(m) : x) << (8 * t);
                            }
                            w[t4] = word;
                        }
                        const int cg = (o.tile_n * BN + c0 + 16 * h) >> 4;
                        if (row < rowsA && cg < cgroups)
                            *reinterpret_cast<uint4*>(prod + ((long(o.z) * cgroups + cg) * rows_pad + row) * 16) =
                                make_uint4(w[0], w[1], w[2], w[3]);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&acc_empty[b]));
            ++j;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
    }
}

__device__ __forceinline__ double oz_frac(double s, double t) {
    double x = s - rint(s);
    x += t;
    return x - rint(x);
}

// C (row, col) = alpha (C_re + i C_im) + beta C: thread (row, h) with row = blockIdx.y * 128 + threadIdx.x / 2
// takes the 4 complex columns 8 blockIdx.x + 4 h .. + 3 (8 bytes of column group blockIdx.x per modulus and
// split: a warp reads 256 contiguous bytes per load)
__global__ void __launch_bounds__(256) k_oz_recombine(int M, int N, int splits, const unsigned char* __restrict__ prod,
                                                      long rows_pad, int cgroups, const int* __restrict__ eA,
                                                      const int* __restrict__ eB, const __grid_constant__ OzConst c,
                                                      double2 alpha, double2 beta, double2* __restrict__ C, long ldc) {
    const int row = blockIdx.y * 128 + (threadIdx.x >> 1);
    const int h = threadIdx.x & 1;
    if (row >= M) return;
    const int cg = blockIdx.x, col0 = 8 * cg + 4 * h;
    if (col0 >= N) return;
    uint2 v[kOzMaxMods];
    // every load of the first split first (independent), then the other splits' residues added byte-wise
#pragma unroll
    for (int l = 0; l < kOzMaxMods; ++l)
        if (l < c.n)
            v[l] = *reinterpret_cast<const uint2*>(prod + ((long(l) * cgroups + cg) * rows_pad + row) * 16 + 8 * h);
    double s[8], t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) s[i] = t[i] = 0.0;
#pragma unroll
    for (int l = 0; l < kOzMaxMods; ++l) {
        if (l >= c.n) break;
        unsigned acc[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = ((i < 4 ? v[l].x : v[l].y) >> (8 * (i & 3))) & 0xFFu;
        for (int sp = 1; sp < splits; ++sp) {
            const long z = long(sp) * c.n + l;
            const uint2 x = *reinterpret_cast<const uint2*>(prod + ((z * cgroups + cg) * rows_pad + row) * 16 + 8 * h);
#pragma unroll
            for (int i = 0; i < 8; ++i) acc[i] += ((i < 4 ? x.x : x.y) >> (8 * (i & 3))) & 0xFFu;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const double cv = double(splits > 1 ? oz_umod(acc[i], c.m[l], c.magic[l]) : acc[i]);
            s[i] = fma(cv, c.wa[l], s[i]);
            t[i] = fma(cv, c.wb[l], t[i]);
        }
    }
    const int ea = eA[row];
    const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const int col = col0 + jj;
        if (col >= N) break;
        const int eb = eB[col];
        double re, im;
        if (ea == kOzNonFinite || eb == kOzNonFinite) {
            re = im = __longlong_as_double(0x7ff8000000000000ll);
        } else {
            const int e = ea + eb;
            re = ldexp(oz_frac(s[2 * jj], t[2 * jj]) * c.mprod, -e);
            im = ldexp(oz_frac(s[2 * jj + 1], t[2 * jj + 1]) * c.mprod, -e);
        }
        double2* cp = C + long(col) * ldc + row;
        double2 o = make_double2(alpha.x * re - alpha.y * im, alpha.x * im + alpha.y * re);
        if (use_beta) {
            const double2 old = *cp;
            o.x += beta.x * old.x - beta.y * old.y;
            o.y += beta.x * old.y + beta.y * old.x;
        }
        *cp = o;
    }
}

// 3-D int8 tensor map over (K', rows, plane): box 128 K bytes x box_rows rows x 1 plane, 128-byte swizzle
CUtensorMap make_map_u8(const void* base, long kr, long rows, long nplanes, long kp, unsigned box_rows) {
    CUtensorMap m;
    const cuuint64_t dims[3] = {cuuint64_t(kr), cuuint64_t(rows), cuuint64_t(nplanes)};
    const cuuint64_t strides[2] = {cuuint64_t(kp), cuuint64_t(kp) * cuuint64_t(rows)};
    const cuuint32_t box[3] = {128, box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box,
                                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    B200_CHECK(r == CUDA_SUCCESS, kInvalidArgument, "cuTensorMapEncodeTiled failed (code " + std::to_string(int(r)) + ")");
    return m;
}

__global__ void k_scale_z(int M, int N, double2 beta, double2* __restrict__ C, long ldc) {
    const long total = long(M) * N;
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const long j = t / M, i = t - j * M;
        double2* p = C + j * ldc + i;
        if (beta.x == 0.0 && beta.y == 0.0) {
            *p = make_double2(0.0, 0.0);
        } else {
            const double2 v = *p;
            *p = make_double2(beta.x * v.x - beta.y * v.y, beta.x * v.y + beta.y * v.x);
        }
    }
}

long round_up(long x, long a) { return (x + a - 1) / a * a; }

void launch_check() {
    note_launch();
    B200_CUDA(cudaGetLastError());
}

// residue form of the columns of X (K x ncols, pitch ld): KIND as in k_oz_res_cols
template <int KIND>
void residues_of_columns(int K, int ncols, const double2* X, long ld, const OzConst& c, OzOperand& out,
                         DeviceArray<double>& part, cudaStream_t s) {
    const int rows = KIND == 0 ? ncols : 2 * ncols;
    out.rows = rows;
    out.kr = 2 * K;
    out.kp = int(round_up(out.kr, 16));
    out.n = c.n;
    out.res.resize(size_t(c.n) * rows * out.kp);
    out.exps.resize(size_t(ncols));
    const int nseg = (K + kOzSeg - 1) / kOzSeg;
    part.resize(size_t(nseg) * ncols);
    B200_CHECK(ncols <= 65535, kInvalidArgument, "int8 GEMM: more than 65535 columns");
    const dim3 grid(nseg, ncols);
    k_oz_absmax_cols<<<grid, 256, 0, s>>>(K, X, ld, part.ptr);
    launch_check();
    k_oz_res_cols<KIND><<<grid, 256, 0, s>>>(K, X, ld, part.ptr, c, out.res.ptr, out.kp, long(rows) * out.kp,
                                             out.exps.ptr);
    launch_check();
}

}  // namespace

int* OzWorkspace::err_ptr() {
    if (!err.ptr) {
        err.resize(1);
        B200_CUDA(cudaMemset(err.ptr, 0, sizeof(int)));
    }
    return err.ptr;
}

int OzWorkspace::read_error(cudaStream_t s) {
    int h = 0;
    if (err.ptr) {
        B200_CUDA(cudaMemcpyAsync(&h, err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
        B200_CUDA(cudaStreamSynchronize(s));
        if (h) B200_CUDA(cudaMemsetAsync(err.ptr, 0, sizeof(int), s));
    }
    return h;
}

void oz_constants(int nmods, long kr, int* mods, double* wa, double* wb, double* mprod, int* q) {
    const OzConst c = oz_const(nmods, kr);
    for (int l = 0; l < nmods; ++l) {
        mods[l] = int(c.m[l]);
        wa[l] = c.wa[l];
        wb[l] = c.wb[l];
    }
    *mprod = c.mprod;
    *q = c.q;
}

void scale_matrix_z(int M, int N, double2 beta, double2* C, int ldc, cudaStream_t s) {
    if (M <= 0 || N <= 0) return;
    B200_CHECK(ldc >= M, kInvalidArgument, "ldc < M");
    const long total = long(M) * N;
    const int blocks = int(std::min<long>((total + 255) / 256, 148L * 8));
    k_scale_z<<<blocks, 256, 0, s>>>(M, N, beta, C, ldc);
    launch_check();
}

void oz_prepare_a(char opa, int M, int K, const double2* A, int lda, int nmods, OzOperand& out, OzWorkspace& w,
                  cudaStream_t s) {
    B200_CHECK(opa == 'N' || opa == 'C', kInvalidArgument, "int8 GEMM: op(A) must be 'N' or 'C'");
    B200_CHECK(M > 0 && K > 0 && A, kInvalidArgument, "int8 GEMM: empty or NULL operand");
    B200_CHECK(opa == 'C' ? lda >= K : lda >= M, kInvalidArgument, "int8 GEMM: lda too small");
    const OzConst c = oz_const(nmods, 2L * K);
    if (opa == 'C') {
        residues_of_columns<0>(K, M, A, lda, c, out, w.part, s);
        return;
    }
    out.rows = M;
    out.kr = 2 * K;
    out.kp = int(round_up(out.kr, 16));
    out.n = nmods;
    out.res.resize(size_t(nmods) * M * out.kp);
    out.exps.resize(size_t(M));
    w.part.resize(size_t(M));
    k_oz_absmax_rows<<<(M + 127) / 128, 128, 0, s>>>(M, K, A, lda, w.part.ptr);
    launch_check();
    B200_CHECK((M + 31) / 32 <= 65535, kInvalidArgument, "int8 GEMM: too many rows");
    k_oz_res_rows<<<dim3((K + 31) / 32, (M + 31) / 32), dim3(32, 8), 0, s>>>(M, K, A, lda, w.part.ptr, c, out.res.ptr,
                                                                            out.kp, long(M) * out.kp, out.exps.ptr);
    launch_check();
}

void oz_zgemm(char opa, int M, int N, int K, double2 alpha, const OzOperand& a, const double2* B, int ldb,
              double2 beta, double2* C, int ldc, OzWorkspace& w, int* err, cudaStream_t s) {
    B200_CHECK(opa == 'N' || opa == 'C', kInvalidArgument, "int8 GEMM: op(A) must be 'N' or 'C'");
    B200_CHECK(M > 0 && N > 0 && K > 0 && B && C, kInvalidArgument, "int8 GEMM: empty or NULL operand");
    B200_CHECK(a.rows == M && a.kr == 2 * K && a.res.ptr, kInvalidArgument,
               "int8 GEMM: op(A) residues do not match M and K");
    B200_CHECK(ldb >= K && ldc >= M, kInvalidArgument, "int8 GEMM: ldb < K or ldc < M");
    const OzConst c = oz_const(a.n, a.kr);
    if (!err) err = w.err_ptr();
    if (opa == 'N') residues_of_columns<1>(K, N, B, ldb, c, w.b, w.part, s);
    else residues_of_columns<2>(K, N, B, ldb, c, w.b, w.part, s);

    // tiles: 128 msub rows of op(A) x BN real columns (BN <= 256, a multiple of 16)
    const int colsB = 2 * N;
    const int tn = (colsB + 255) / 256;
    const int BN = int(round_up((colsB + tn - 1) / tn, 16));
    const int tm128 = (M + 127) / 128;
    const int nk = (a.kr + 127) / 128;
    int sms = 148, dev = 0;
    B200_CUDA(cudaGetDevice(&dev));
    B200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // K splits: within the exact int32 range; among those, the fewest waves of tiles times K blocks per tile
    // (plus a few blocks' worth per tile for its epilogue and pipeline fill) over the SMs
    const long tiles128 = long(tm128) * tn * a.n;
    const int msub = (tm128 >= 2 && nk >= 64) ? 2 : 1;  // 256-row tiles for long K (streamed B' read half as often)
    const long tiles_sp = (long(tm128 + msub - 1) / msub) * tn * a.n;
    int splits = (nk + kOzMaxKbPerSplit - 1) / kOzMaxKbPerSplit;
    {
        double best = 1e300;
        int bs = splits;
        for (int sp = splits; sp <= 64 && sp <= nk; ++sp) {
            const long per_sp = (nk + sp - 1) / sp;
            if (sp > splits && per_sp < 16) break;
            const long waves = (tiles_sp * sp + sms - 1) / sms;
            const double cost = double(waves) * double(per_sp + 4) + 0.02 * sp;
            if (cost < best - 1e-9) {
                best = cost;
                bs = sp;
            }
        }
        splits = bs;
    }
    (void)tiles128;
    const int per = (nk + splits - 1) / splits;
    splits = (nk + per - 1) / per;
    // B' of one (plane, column tile) resident in shared memory when it leaves room for 3 stages of A; else
    // streamed with A, and long K ranges take 256-row tiles (two accumulators: half the re-reads of B')
    const int b_box = BN * 128;
    const int fixed = 1024 + 256;  // alignment slack, barriers
    OzSched sc{tm128, tn, a.n * splits, per, nk, 1, 2, false};
    int stages;
    if (tn <= sms && long(per) * b_box + 3L * kOzATile + fixed <= kOzSmem) {
        sc.resident = true;
        stages = int((kOzSmem - fixed - long(per) * b_box) / kOzATile);
    } else {
        sc.msub = msub;
        sc.tm = (tm128 + msub - 1) / msub;
        stages = (kOzSmem - fixed) / (sc.msub * kOzATile + b_box);
    }
    if (stages > 8) stages = 8;
    sc.nbuf = sc.msub * BN <= 256 ? 2 : 1;
    const long T = long(sc.tm) * tn * sc.nz;
    int grid = int(T < sms ? T : sms);
    if (sc.resident) grid = int(std::min<long>(long(sms / tn) * tn, long(sc.tm) * sc.nz * tn));
    const long rows_pad = M;
    const int cgroups = int(round_up(colsB, 16) / 16);
    w.prod.resize(size_t(sc.nz) * cgroups * rows_pad * 16);
    const CUtensorMap mA = make_map_u8(a.res.ptr, a.kr, M, a.n, a.kp, 128);
    const CUtensorMap mB = make_map_u8(w.b.res.ptr, w.b.kr, colsB, a.n, w.b.kp, unsigned(BN));
    OzMods md{};
    for (int l = 0; l < a.n; ++l) {
        md.m[l] = c.m[l];
        md.magic[l] = c.magic[l];
        md.c31[l] = c.c31[l];
    }
    static std::once_flag once;
    std::call_once(once, [] {
        B200_CUDA(cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem));
    });
    k_oz_gemm<<<grid, kOzThreads, kOzSmem, s>>>(mA, mB, M, BN, stages, a.n, sc, md, w.prod.ptr, rows_pad, cgroups,
                                                err, tc_wait_limit_ns());
    launch_check();
    B200_CHECK((M + 127) / 128 <= 65535, kInvalidArgument, "int8 GEMM: too many rows");
    k_oz_recombine<<<dim3(cgroups, (M + 127) / 128), 256, 0, s>>>(M, N, splits, w.prod.ptr, rows_pad, cgroups,
                                                                  a.exps.ptr, w.b.exps.ptr, c, alpha, beta, C, ldc);
    launch_check();
}

}  // namespace b200
