// FP64 complex GEMM on the int8 tensor cores (tcgen05 kind::i8), exact modular emulation (gemm_oz.cu).
//
// Every real row of op(A) and every real column of B is scaled by a power of two and rounded to an integer
// (its largest entry below 2^q, q >= 52 for 16 moduli and K' <= 2^18); the integer matrices are reduced
// modulo n pairwise coprime moduli m_l <= 256 (signed residues, int8), one exact int8 GEMM per modulus
// (int32 accumulation), and the integer product is recombined from its n residues by the Chinese
// remainder theorem, then scaled back.
// With n = 16 an entry's error is of the order of an FP64 GEMM's.  NaN or infinite entries in a row of
// op(A) or a column of B make the entries of C that they reach NaN.
#pragma once
#include <cuda_runtime.h>

#include "common.h"

namespace b200 {

constexpr int kOzMinMods = 12;
constexpr int kOzMaxMods = 16;

// One operand in residue form: `rows` real rows of `kr` entries (K-major), stored as n int8 planes of
// rows x kp bytes (kp = kr rounded up to 16), and one power-of-two exponent per row group (a row of
// op(A); a complex column of B, which gives two real rows).
struct OzOperand {
    DeviceArray<signed char> res;
    DeviceArray<int> exps;
    int rows = 0, kr = 0, kp = 0, n = 0;
    size_t device_bytes() const { return res.n + exps.n * sizeof(int); }
};

// Scratch of one caller: the per-call operand residues, norm partial sums, the residues of the
// per-modulus products and an error word (set when a bounded wait inside the GEMM kernel runs out).
struct OzWorkspace {
    OzOperand a, b;
    DeviceArray<double> part;
    DeviceArray<unsigned char> prod;
    DeviceArray<int> err;
    int* err_ptr();  // allocated and zeroed at first use
    int read_error(cudaStream_t s);
    size_t device_bytes() const {
        return a.device_bytes() + b.device_bytes() + part.n * sizeof(double) + prod.n + err.n * sizeof(int);
    }
};

// op(A) of C = alpha op(A) B + beta C in residue form: opa 'N' takes the rows of A (M x K, column-major,
// pitch lda), 'C' the columns of A (K x M) conjugated.  nmods in [kOzMinMods, kOzMaxMods].
void oz_prepare_a(char opa, int M, int K, const double2* A, int lda, int nmods, OzOperand& out, OzWorkspace& w,
                  cudaStream_t s);

// C (M x N) = alpha op(A) B + beta C, complex128 column-major, op(A) given in residue form (oz_prepare_a
// with the same opa, M and K); B is K x N with pitch ldb.  beta = 0: C is not read.  err: device error word
// of the GEMM kernel's bounded waits (nullptr: the workspace's own).
void oz_zgemm(char opa, int M, int N, int K, double2 alpha, const OzOperand& a, const double2* B, int ldb,
              double2 beta, double2* C, int ldc, OzWorkspace& w, int* err, cudaStream_t s);

// C = beta C (beta = 0: C = 0 without reading it), complex128 column-major M x N
void scale_matrix_z(int M, int N, double2 beta, double2* C, int ldc, cudaStream_t s);

// host copies of the recombination constants for n moduli (tests): the moduli, the weights w_l / M as
// wa + wb (wa with 40 fraction bits), M rounded to a double, and the scale exponent q for real rows of
// length kr (every row's largest magnitude is brought below 2^q)
void oz_constants(int nmods, long kr, int* mods, double* wa, double* wb, double* mprod, int* q);

}  // namespace b200
