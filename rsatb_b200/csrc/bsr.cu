// Device-resident BSR matrices: the vbcsr BlockSpMat<T> subset the hot path
// needs (construct/assemble, adjoint, precision copy, value updates).
#include "common.cuh"

#include <algorithm>
#include <vector>

namespace rsatb_b200 {
namespace {

// out block `dst[k]` = conj(transpose(in block `src_of[k]`)), one thread per
// element.  T is the real component type; C selects complex values.
template <typename T, bool C>
__global__ void bsr_adjoint_values(const T* __restrict__ in, T* __restrict__ out,
                                   const int64_t* __restrict__ src_of, int64_t nnzb, int b) {
    const int64_t bb = int64_t(b) * b;
    const int64_t total = nnzb * bb;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t k = e / bb;
        const int rc = int(e - k * bb);
        const int r = rc / b, c = rc % b;
        const int64_t src = src_of[k] * bb + int64_t(c) * b + r;
        if (C) {
            out[2 * e] = in[2 * src];
            out[2 * e + 1] = -in[2 * src + 1];
        } else {
            out[e] = in[src];
        }
    }
}

template <typename T>
__global__ void negate_values(T* __restrict__ v, int64_t n) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x)
        v[e] = -v[e];
}

template <typename TI, typename TO>
__global__ void cast_values(const TI* __restrict__ in, TO* __restrict__ out, int64_t n) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x)
        out[e] = static_cast<TO>(in[e]);
}

int grid_for(const rsatb_context* ctx, int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    int64_t cap = int64_t(ctx->sm_count) * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return int(g);
}

}  // namespace

void free_matrix(rsatb_bsr_matrix* A) {
    if (!A) return;
    cudaSetDevice(A->device);
    if (A->row_ptr) cudaFree(A->row_ptr);
    if (A->col_ind) cudaFree(A->col_ind);
    if (A->values) cudaFree(A->values);
    delete A;
}

// Allocates an empty matrix shell with device arrays of the right size.
int alloc_matrix(int device, int nbr, int nbc, int b, int64_t nnzb, int dtype, unsigned flags,
                 rsatb_bsr_matrix** out) {
    auto* A = new rsatb_bsr_matrix();
    A->device = device;
    A->n_block_rows = nbr;
    A->n_block_cols = nbc;
    A->block_size = b;
    A->nnz_blocks = nnzb;
    A->dtype = dtype;
    A->flags = flags & RSATB_BSR_IMAGINARY_UNIT;
    cudaError_t e1 = cudaMalloc(&A->row_ptr, sizeof(int32_t) * (size_t(nbr) + 1));
    cudaError_t e2 = cudaMalloc(&A->col_ind, sizeof(int32_t) * size_t(std::max<int64_t>(nnzb, 1)));
    cudaError_t e3 = cudaMalloc(&A->values, dtype_size(dtype) * size_t(std::max<int64_t>(nnzb, 1)) *
                                                size_t(b) * size_t(b));
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        free_matrix(A);
        return set_error(RSATB_OUT_OF_MEMORY, "BSR allocation of %lld blocks of %dx%d failed",
                         (long long)nnzb, b, b);
    }
    *out = A;
    return RSATB_SUCCESS;
}

}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" {

int rsatb_bsr_create(rsatb_ctx_t ctx, int n_block_rows, int n_block_cols, int block_size,
                     int64_t nnz_blocks, const int32_t* row_ptr, const int32_t* col_ind,
                     const void* values, rsatb_dtype dtype, unsigned flags, rsatb_bsr_t* out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!out) return set_error(RSATB_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    if (n_block_rows < 0 || n_block_cols < 0 || block_size <= 0 || block_size > 16 ||
        nnz_blocks < 0 || !dtype_valid(dtype))
        return set_error(RSATB_INVALID_ARGUMENT,
                         "bsr_create: bad shape (rows %d cols %d b %d nnzb %lld dtype %d); "
                         "block sizes 1..16 are supported",
                         n_block_rows, n_block_cols, block_size, (long long)nnz_blocks, (int)dtype);
    if (nnz_blocks > 0 && (!row_ptr || !col_ind || !values))
        return set_error(RSATB_INVALID_ARGUMENT, "bsr_create: null array");
    if ((flags & RSATB_BSR_IMAGINARY_UNIT) && dtype_is_complex(dtype))
        return set_error(RSATB_INVALID_ARGUMENT,
                         "bsr_create: the imaginary-unit flag needs real values");
    const bool on_dev = flags & RSATB_BSR_DEVICE_POINTERS;

    // Validate the pattern on the host (a bad index would read out of bounds
    // in every later kernel).
    std::vector<int32_t> h_ptr(size_t(n_block_rows) + 1);
    std::vector<int32_t> h_ind(static_cast<size_t>(nnz_blocks));
    if (on_dev) {
        RSATB_CUDA_TRY(cudaMemcpy(h_ptr.data(), row_ptr, sizeof(int32_t) * h_ptr.size(),
                                  cudaMemcpyDeviceToHost));
        if (nnz_blocks)
            RSATB_CUDA_TRY(cudaMemcpy(h_ind.data(), col_ind, sizeof(int32_t) * h_ind.size(),
                                      cudaMemcpyDeviceToHost));
    } else {
        if (row_ptr) std::copy(row_ptr, row_ptr + h_ptr.size(), h_ptr.begin());
        else h_ptr.assign(h_ptr.size(), 0);
        if (nnz_blocks) std::copy(col_ind, col_ind + h_ind.size(), h_ind.begin());
    }
    if (h_ptr[0] != 0 || h_ptr[n_block_rows] != nnz_blocks)
        return set_error(RSATB_INVALID_ARGUMENT, "bsr_create: row_ptr must run 0..nnz_blocks");
    int max_row = 0;
    for (int i = 0; i < n_block_rows; ++i) {
        if (h_ptr[i + 1] < h_ptr[i])
            return set_error(RSATB_INVALID_ARGUMENT, "bsr_create: row_ptr decreases at row %d", i);
        max_row = std::max(max_row, h_ptr[i + 1] - h_ptr[i]);
        for (int k = h_ptr[i]; k < h_ptr[i + 1]; ++k) {
            if (h_ind[k] < 0 || h_ind[k] >= n_block_cols)
                return set_error(RSATB_INVALID_ARGUMENT,
                                 "bsr_create: column %d out of range in row %d", h_ind[k], i);
        }
    }

    rsatb_bsr_matrix* A = nullptr;
    RSATB_TRY(alloc_matrix(ctx->device, n_block_rows, n_block_cols, block_size, nnz_blocks, dtype,
                           flags, &A));
    A->max_row_blocks = max_row;
    const size_t vbytes = dtype_size(dtype) * size_t(nnz_blocks) * block_size * block_size;
    cudaError_t err = cudaMemcpy(A->row_ptr, h_ptr.data(), sizeof(int32_t) * h_ptr.size(),
                                 cudaMemcpyHostToDevice);
    if (err == cudaSuccess && nnz_blocks)
        err = cudaMemcpy(A->col_ind, h_ind.data(), sizeof(int32_t) * h_ind.size(),
                         cudaMemcpyHostToDevice);
    if (err == cudaSuccess && nnz_blocks)
        err = cudaMemcpy(A->values, values, vbytes, cudaMemcpyDefault);
    if (err != cudaSuccess) {
        free_matrix(A);
        return set_error(RSATB_CUDA_ERROR, "bsr_create upload: %s", cudaGetErrorString(err));
    }
    *out = A;
    return RSATB_SUCCESS;
}

int rsatb_bsr_destroy(rsatb_bsr_t A) {
    clear_error();
    free_matrix(A);
    return RSATB_SUCCESS;
}

int rsatb_bsr_info(rsatb_bsr_t A, int* n_block_rows, int* n_block_cols, int* block_size,
                   int64_t* nnz_blocks, int* dtype, unsigned* flags) {
    clear_error();
    RSATB_TRY(check_bsr(A, "bsr_info"));
    if (n_block_rows) *n_block_rows = A->n_block_rows;
    if (n_block_cols) *n_block_cols = A->n_block_cols;
    if (block_size) *block_size = A->block_size;
    if (nnz_blocks) *nnz_blocks = A->nnz_blocks;
    if (dtype) *dtype = A->dtype;
    if (flags) *flags = A->flags;
    return RSATB_SUCCESS;
}

void* rsatb_bsr_values(rsatb_bsr_t A) { return A ? A->values : nullptr; }

int rsatb_bsr_set_values(rsatb_ctx_t ctx, rsatb_bsr_t A, const void* values, unsigned flags) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_TRY(check_bsr(A, "bsr_set_values"));
    if (!values && A->nnz_blocks) return set_error(RSATB_INVALID_ARGUMENT, "null values");
    (void)flags;  // cudaMemcpyDefault infers the direction
    const size_t vbytes =
        dtype_size(A->dtype) * size_t(A->nnz_blocks) * A->block_size * A->block_size;
    if (vbytes)
        RSATB_CUDA_TRY(cudaMemcpyAsync(A->values, values, vbytes, cudaMemcpyDefault, ctx->stream));
    return RSATB_SUCCESS;
}

int rsatb_bsr_pattern(rsatb_ctx_t ctx, rsatb_bsr_t A, int32_t* row_ptr, int32_t* col_ind) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_TRY(check_bsr(A, "bsr_pattern"));
    if (!row_ptr || (A->nnz_blocks && !col_ind))
        return set_error(RSATB_INVALID_ARGUMENT, "null output array");
    RSATB_CUDA_TRY(cudaMemcpyAsync(row_ptr, A->row_ptr,
                                   sizeof(int32_t) * (size_t(A->n_block_rows) + 1),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    if (A->nnz_blocks)
        RSATB_CUDA_TRY(cudaMemcpyAsync(col_ind, A->col_ind, sizeof(int32_t) * size_t(A->nnz_blocks),
                                       cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return RSATB_SUCCESS;
}

int rsatb_bsr_adjoint(rsatb_ctx_t ctx, rsatb_bsr_t A, rsatb_bsr_t* out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_TRY(check_bsr(A, "bsr_adjoint"));
    if (!out) return set_error(RSATB_INVALID_ARGUMENT, "null output pointer");
    const int nbr = A->n_block_rows, nbc = A->n_block_cols, b = A->block_size;
    const int64_t nnzb = A->nnz_blocks;
    std::vector<int32_t> ptr(static_cast<size_t>(nbr) + 1), ind(static_cast<size_t>(nnzb));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpy(ptr.data(), A->row_ptr, sizeof(int32_t) * ptr.size(),
                              cudaMemcpyDeviceToHost));
    if (nnzb)
        RSATB_CUDA_TRY(cudaMemcpy(ind.data(), A->col_ind, sizeof(int32_t) * ind.size(),
                                  cudaMemcpyDeviceToHost));
    // Counting sort by column: rows of A^H are columns of A, and walking A's
    // rows in order keeps each new row's columns sorted.
    std::vector<int32_t> tptr(static_cast<size_t>(nbc) + 1, 0), tind(static_cast<size_t>(nnzb));
    std::vector<int64_t> src_of(static_cast<size_t>(nnzb));
    for (int64_t k = 0; k < nnzb; ++k) tptr[ind[k] + 1]++;
    for (int j = 0; j < nbc; ++j) tptr[j + 1] += tptr[j];
    std::vector<int32_t> fill(tptr.begin(), tptr.end() - 1);
    int max_row = 0;
    for (int i = 0; i < nbr; ++i) {
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
            const int j = ind[k];
            const int dst = fill[j]++;
            tind[dst] = i;
            src_of[dst] = k;
        }
    }
    for (int j = 0; j < nbc; ++j) max_row = std::max(max_row, tptr[j + 1] - tptr[j]);

    rsatb_bsr_matrix* T = nullptr;
    RSATB_TRY(alloc_matrix(ctx->device, nbc, nbr, b, nnzb, A->dtype, A->flags, &T));
    T->max_row_blocks = max_row;
    int64_t* d_src = nullptr;
    cudaError_t err = cudaMemcpy(T->row_ptr, tptr.data(), sizeof(int32_t) * tptr.size(),
                                 cudaMemcpyHostToDevice);
    if (err == cudaSuccess && nnzb)
        err = cudaMemcpy(T->col_ind, tind.data(), sizeof(int32_t) * tind.size(),
                         cudaMemcpyHostToDevice);
    if (err == cudaSuccess && nnzb) err = cudaMalloc(&d_src, sizeof(int64_t) * nnzb);
    if (err == cudaSuccess && nnzb)
        err = cudaMemcpy(d_src, src_of.data(), sizeof(int64_t) * nnzb, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        free_matrix(T);
        if (d_src) cudaFree(d_src);
        return set_error(RSATB_CUDA_ERROR, "bsr_adjoint: %s", cudaGetErrorString(err));
    }
    if (nnzb) {
        const int threads = 256;
        const int grid = grid_for(ctx, nnzb * b * b, threads);
        switch (A->dtype) {
            case RSATB_F64:
                bsr_adjoint_values<double, false><<<grid, threads, 0, ctx->stream>>>(
                    (const double*)A->values, (double*)T->values, d_src, nnzb, b);
                break;
            case RSATB_F32:
                bsr_adjoint_values<float, false><<<grid, threads, 0, ctx->stream>>>(
                    (const float*)A->values, (float*)T->values, d_src, nnzb, b);
                break;
            case RSATB_C128:
                bsr_adjoint_values<double, true><<<grid, threads, 0, ctx->stream>>>(
                    (const double*)A->values, (double*)T->values, d_src, nnzb, b);
                break;
            case RSATB_C64:
                bsr_adjoint_values<float, true><<<grid, threads, 0, ctx->stream>>>(
                    (const float*)A->values, (float*)T->values, d_src, nnzb, b);
                break;
        }
        err = cudaGetLastError();
        if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
        ctx->launches++;
        cudaFree(d_src);
        if (err != cudaSuccess) {
            free_matrix(T);
            return set_error(RSATB_CUDA_ERROR, "bsr_adjoint kernel: %s", cudaGetErrorString(err));
        }
    }
    // The adjoint of i*W (W real) is -i*W^T: the flag stays and the
    // transposed values change sign.
    if ((A->flags & RSATB_BSR_IMAGINARY_UNIT) && nnzb) {
        const int64_t n = nnzb * b * b;
        const int threads = 256;
        const int grid = grid_for(ctx, n, threads);
        if (A->dtype == RSATB_F64)
            negate_values<double><<<grid, threads, 0, ctx->stream>>>((double*)T->values, n);
        else
            negate_values<float><<<grid, threads, 0, ctx->stream>>>((float*)T->values, n);
        err = cudaGetLastError();
        ctx->launches++;
        if (err != cudaSuccess) {
            free_matrix(T);
            return set_error(RSATB_CUDA_ERROR, "bsr_adjoint negate: %s", cudaGetErrorString(err));
        }
    }
    *out = T;
    return RSATB_SUCCESS;
}

int rsatb_bsr_convert(rsatb_ctx_t ctx, rsatb_bsr_t A, rsatb_dtype dtype, rsatb_bsr_t* out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_TRY(check_bsr(A, "bsr_convert"));
    if (!out) return set_error(RSATB_INVALID_ARGUMENT, "null output pointer");
    if (!dtype_valid(dtype) || dtype_is_complex(dtype) != dtype_is_complex(A->dtype))
        return set_error(RSATB_INVALID_ARGUMENT,
                         "bsr_convert: only the precision may change (dtype %d -> %d)", A->dtype,
                         (int)dtype);
    const int b = A->block_size;
    rsatb_bsr_matrix* T = nullptr;
    RSATB_TRY(alloc_matrix(ctx->device, A->n_block_rows, A->n_block_cols, b, A->nnz_blocks, dtype,
                           A->flags, &T));
    T->max_row_blocks = A->max_row_blocks;
    cudaError_t err = cudaMemcpyAsync(T->row_ptr, A->row_ptr,
                                      sizeof(int32_t) * (size_t(A->n_block_rows) + 1),
                                      cudaMemcpyDeviceToDevice, ctx->stream);
    if (err == cudaSuccess && A->nnz_blocks)
        err = cudaMemcpyAsync(T->col_ind, A->col_ind, sizeof(int32_t) * size_t(A->nnz_blocks),
                              cudaMemcpyDeviceToDevice, ctx->stream);
    if (err != cudaSuccess) {
        free_matrix(T);
        return set_error(RSATB_CUDA_ERROR, "bsr_convert: %s", cudaGetErrorString(err));
    }
    const int64_t n = A->nnz_blocks * b * b * (dtype_is_complex(dtype) ? 2 : 1);
    if (n) {
        const int threads = 256;
        const int grid = grid_for(ctx, n, threads);
        const bool in_d = dtype_is_double(A->dtype), out_d = dtype_is_double(dtype);
        if (in_d && out_d)
            cast_values<double, double><<<grid, threads, 0, ctx->stream>>>(
                (const double*)A->values, (double*)T->values, n);
        else if (in_d && !out_d)
            cast_values<double, float><<<grid, threads, 0, ctx->stream>>>(
                (const double*)A->values, (float*)T->values, n);
        else if (!in_d && out_d)
            cast_values<float, double><<<grid, threads, 0, ctx->stream>>>(
                (const float*)A->values, (double*)T->values, n);
        else
            cast_values<float, float><<<grid, threads, 0, ctx->stream>>>(
                (const float*)A->values, (float*)T->values, n);
        err = cudaGetLastError();
        ctx->launches++;
        if (err != cudaSuccess) {
            free_matrix(T);
            return set_error(RSATB_CUDA_ERROR, "bsr_convert kernel: %s", cudaGetErrorString(err));
        }
    }
    *out = T;
    return RSATB_SUCCESS;
}

}  // extern "C"
