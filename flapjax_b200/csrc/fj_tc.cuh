// fj_tc.cuh -- tensor-core (tcgen05, TF32 operands, FP32 accumulation) building blocks of
// the mixed-precision factorisation.
#pragma once

#include "fj_common.cuh"

namespace fj {

// C <- alpha A B + beta C; A (m x k, lda), B (k x n, ldb), C (m x n, ldc) row-major FP32.
// passes = 1: TF32 products; passes = 3: hi/lo split, close to FP32 accuracy.  C may be the
// memory of B when m <= 128 (each CTA then reads only the B columns it writes).  beta = 0
// never reads C.  *d_err (device int) is set to 1 if a bounded device wait expired.
int tc_gemm_tf32(const float* a, int lda, const float* b, int ldb, float* c, int ldc, int m, int n, int k,
                 float alpha, float beta, int passes, int* d_err, cudaStream_t s);

// The same product fed by TMA (the factorisation's form): the operands are first split
// into scratch (tc_gemm_scratch_floats of it, 16-byte aligned), so C may overlap A or B
// anywhere.  Without enough scratch, or where the driver has no tensor-map encoder, it
// runs tc_gemm_tf32.
size_t tc_gemm_scratch_floats(int m, int n, int k, int passes);
int tc_gemm_tf32_tma(const float* a, int lda, const float* b, int ldb, float* c, int ldc, int m, int n, int k,
                     float alpha, float beta, int passes, float* scratch, size_t scratch_floats, int* d_err,
                     cudaStream_t s);

// Inverses of the 128 x 128 diagonal blocks b0 .. b0+nb-1 of packed n x n LU factors (the
// last block of the matrix may be smaller): of the unit lower triangle, or (upper) of the
// upper triangle with its diagonal.  Block b goes to out + 128*128*b, row-major, zero
// outside the block.
int tri_inverse32_blocks(const float* lu, int n, int b0, int nb, bool upper, float* out, cudaStream_t s);

}  // namespace fj
