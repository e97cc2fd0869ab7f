// FP64 matrix product C = A B^T emulated on the int8 tensor cores (tcgen05.mma kind::i8).
//
// Each row of A and of B is split into `slices` signed 8-bit digit planes over one power-of-two
// scale per row (an Ozaki-type splitting: Ozaki, Ogita, Oishi & Rump, Numer. Algorithms 59
// (2012) 95-118): x = 2^(e-7) sum_s d_s 128^-s with d_0 in [-127, 127], d_s in [-64, 64] for
// s >= 1 (round-to-nearest digits, so the dropped remainder is at most 2^(e-7*slices-1)).  The
// products of digit planes with s + t = level share one scale, so each level is one exact int32
// accumulation over K on the tensor cores; the levels 0 .. slices-1 are summed in FP64.  The
// result differs from a correctly rounded FP64 product by about 2^(1-7*slices) times
// max_k |A_ik| sum_k |B_jk| + sum_k |A_ik| max_k |B_jk| (slices = 7: ~3.6e-15 of that scale).
#pragma once
#include <cstdint>

namespace dgemm_i8 {

constexpr int kMaxSlices = 8;

// Workspace bytes for an m x n x k product with `slices` digit planes and `split` K ranges
// (split <= 0: chosen by the library); < 0 for invalid sizes.
int64_t workspace_bytes(int m, int n, int k, int slices, int split);

// C[i * ldc + j] = sum_k op(A)[i, k] op(B)[j, k] with op(A)[i, k] = A[i * lda + k], or A[k * lda + i]
// when trans_a (A stored [k, m]), the same for B (device pointers).  Workspace:
// >= workspace_bytes(m, n, k, slices, split) bytes, 256-byte aligned.  Returns a DISCOEB_* status;
// a kernel whose bounded waits ran out (never in a correct launch) makes C NaN.
int32_t run(int m, int n, int k, const double* A, int64_t lda, bool trans_a, const double* B, int64_t ldb,
            bool trans_b, double* C, int64_t ldc, int slices, int split, char* ws, int64_t ws_bytes, void* stream);

}  // namespace dgemm_i8
