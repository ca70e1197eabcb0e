// Sliced int8 tensor-core GEMM (tc_gemm.cu): FP64-accurate products on the
// tcgen05 tensor cores, used by the mixed form of the integral stages.
#pragma once
#include "gli_internal.cuh"

namespace gli {

// S int8 slices of `batches` row blocks of `rows` rows (one block's rows count),
// K padded to Kp (multiple of 32), slice-major, one exponent per row
struct SlicedMatrix {
    DevBuf<int8_t> data;
    DevBuf<int> e;
    i64 rows = 0, Kp = 0, batches = 1;
    int slices = 0;
    i64 slice_stride() const { return rows * Kp * batches; }
};

// slice rows of an FP64 matrix (rows x K per batch, row stride ld, batch stride bs)
// nslices = 5 (the mixed form: ~1e-9 Ha on the integral values) or 7 (FP64-level)
void slice_rows(const double* src, i64 rows, int K, i64 ld, i64 bs, int batches, int nslices, SlicedMatrix& out,
                cudaStream_t s);

// C[b] (+)= A[b] B[b]^T; ragged B batches via b_row0/b_rows and output column
// offsets c_col0 (device arrays, or NULL for uniform batches)
void tc_gemm_sliced(const SlicedMatrix& A, const SlicedMatrix& B, int n_max, double* C, i64 rs, i64 cs, i64 bs,
                    int batches, const int* b_row0, const int* b_rows, const int* c_col0, bool accumulate,
                    cudaStream_t s);

}  // namespace gli
