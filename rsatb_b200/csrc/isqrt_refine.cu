// Global sparse Newton-Schulz refinement of S^-1/2 on the device
// (rsatb::calc::inverse_sqrt, rsatb/calc/isqrtm.hpp:262-900): the seed Z
// (the graph-local factor) is refined by
//
//     X = Z^H S Z,   P = 1.875 I - 1.25 X + 0.375 X^2,   Z <- Z P
//
// with every product a block-sparse matrix product (SpGEMM) whose blocks of
// Frobenius norm below sptol are dropped, X advanced either by reformation
// or by propagation P X P, and the reference's stopping rules.
//
// SpGEMM C = alpha A B + beta D + gamma I, FP64, uniform b x b blocks:
//
//  * symbolic: one CTA per output row builds the row's column set as a
//    bitmap in shared memory (one bit per block column: the union of B's
//    rows k over A's row i, D's row i and the diagonal), counts it, and a
//    second pass writes the set bits in order: sorted column indices with
//    no sort.  Row offsets are summed on the host between the passes.
//  * numeric: one warp per output block (i, j) walks A's row i in chunks of
//    32 columns; each lane binary-searches its column k in row j of B^T (the
//    transpose holds B_kj^T at (j, k), so for a symmetric B it is B itself),
//    and the matched pairs, taken in ascending k, are multiplied into the
//    block with each lane owning two of its b*b elements: a fixed summation
//    order, hence deterministic.
//  * drop: the finished blocks (symmetrised as (C + C^T)/2 where the result
//    is Hermitian by construction: X, X^2, P X P) whose Frobenius norm is
//    below sptol are removed by a per-row ballot compaction.
//
// The transposes Z^H and (S Z)^T come from rsatb_bsr_adjoint.
#include "cheb_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a);

namespace {

constexpr int kRowThreads = 256;
constexpr size_t kMaxBitmapBytes = 200 * 1024;

struct MatDel {
    void operator()(rsatb_bsr_matrix* m) const { free_matrix(m); }
};
using Mat = std::unique_ptr<rsatb_bsr_matrix, MatDel>;

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

int dev_alloc(DevBuf& b, size_t bytes) {
    RSATB_CUDA_TRY(cudaMalloc(&b.p, bytes > 0 ? bytes : 16));
    return RSATB_SUCCESS;
}

int grid_cap(const rsatb_context* ctx, int64_t items, int per_cta) {
    int64_t g = (items + per_cta - 1) / per_cta;
    const int64_t cap = int64_t(ctx->sm_count) * 32;
    if (g > cap) g = cap;
    return int(g < 1 ? 1 : g);
}

// ------------------------------------------------------------- symbolic

struct Pattern {
    const int32_t* rp;
    const int32_t* ci;
};

__device__ void row_bitmap(unsigned* bm, int words, int i, Pattern A, Pattern B, Pattern D,
                           bool diag) {
    for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int p = A.rp[i] + warp; p < A.rp[i + 1]; p += nw) {
        const int k = A.ci[p];
        for (int q = B.rp[k] + lane; q < B.rp[k + 1]; q += 32) {
            const int j = B.ci[q];
            atomicOr(&bm[j >> 5], 1u << (j & 31));
        }
    }
    if (D.rp)
        for (int q = D.rp[i] + threadIdx.x; q < D.rp[i + 1]; q += blockDim.x) {
            const int j = D.ci[q];
            atomicOr(&bm[j >> 5], 1u << (j & 31));
        }
    if (diag && threadIdx.x == 0) atomicOr(&bm[i >> 5], 1u << (i & 31));
    __syncthreads();
}

__global__ void __launch_bounds__(kRowThreads) sym_count(int n_rows, int words, Pattern A,
                                                         Pattern B, Pattern D, int diag,
                                                         int32_t* counts) {
    extern __shared__ unsigned bm[];
    __shared__ int part[kRowThreads / 32];
    for (int i = blockIdx.x; i < n_rows; i += gridDim.x) {
        row_bitmap(bm, words, i, A, B, D, diag != 0);
        int c = 0;
        for (int w = threadIdx.x; w < words; w += blockDim.x) c += __popc(bm[w]);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int w = 0; w < int(blockDim.x >> 5); ++w) s += part[w];
            counts[i] = s;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kRowThreads) sym_fill(int n_rows, int words, Pattern A,
                                                        Pattern B, Pattern D, int diag,
                                                        const int32_t* rp_out, int32_t* ci_out) {
    extern __shared__ unsigned bm[];
    __shared__ int offs[kRowThreads];
    const int wpt = (words + blockDim.x - 1) / blockDim.x;
    for (int i = blockIdx.x; i < n_rows; i += gridDim.x) {
        row_bitmap(bm, words, i, A, B, D, diag != 0);
        const int w0 = threadIdx.x * wpt, w1 = min(words, w0 + wpt);
        int c = 0;
        for (int w = w0; w < w1; ++w) c += __popc(bm[w]);
        offs[threadIdx.x] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int t = 0; t < int(blockDim.x); ++t) {
                const int v = offs[t];
                offs[t] = s;
                s += v;
            }
        }
        __syncthreads();
        int pos = rp_out[i] + offs[threadIdx.x];
        for (int w = w0; w < w1; ++w) {
            unsigned bits = bm[w];
            while (bits) {
                const int t = __ffs(bits) - 1;
                bits &= bits - 1;
                ci_out[pos++] = w * 32 + t;
            }
        }
        __syncthreads();
    }
}

__global__ void rows_of_blocks(int n_rows, const int32_t* rp, int32_t* row_of) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_rows; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) row_of[k] = i;
}

// Position of column j in ci[lo, hi) (sorted), or -1.
__device__ __forceinline__ int find_col(const int32_t* ci, int lo, int hi, int j) {
    int a = lo, b = hi;
    while (a < b) {
        const int m = (a + b) >> 1;
        if (ci[m] < j) a = m + 1;
        else b = m;
    }
    return (a < hi && ci[a] == j) ? a : -1;
}

// ------------------------------------------------------------- numeric

struct Vals {
    const int32_t* rp;
    const int32_t* ci;
    const double* v;
};

// BS: compile-time block size (0: runtime b).  Warp per output block.
template <int BS>
__global__ void __launch_bounds__(256) spgemm_numeric(int64_t nnz_c, int b_rt,
                                                      const int32_t* row_of, const int32_t* cci,
                                                      double* cv, Vals A, Vals BT, Vals D,
                                                      double alpha, double beta, double gamma) {
    const int b = BS ? BS : b_rt;
    const int bb = b * b;
    const int lane = threadIdx.x & 31;
    const int e0 = lane, e1 = lane + 32;
    const int r0 = e0 / b, c0 = e0 % b, r1 = e1 / b, c1 = e1 % b;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t e = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; e < nnz_c;
         e += warps) {
        const int i = row_of[e], j = cci[e];
        const int a0 = A.rp[i], a1 = A.rp[i + 1];
        const int t0 = BT.rp[j], t1 = BT.rp[j + 1];
        double acc0 = 0.0, acc1 = 0.0;
        for (int base = a0; base < a1; base += 32) {
            const int p = base + lane;
            int q = -1;
            if (p < a1) q = find_col(BT.ci, t0, t1, A.ci[p]);
            unsigned mask = __ballot_sync(0xffffffffu, q >= 0);
            while (mask) {
                const int src = __ffs(mask) - 1;
                mask &= mask - 1;
                const int pk = __shfl_sync(0xffffffffu, p, src);
                const int qk = __shfl_sync(0xffffffffu, q, src);
                const double* Ab = A.v + int64_t(pk) * bb;
                const double* Tb = BT.v + int64_t(qk) * bb;
                if (e0 < bb) {
#pragma unroll
                    for (int m = 0; m < (BS ? BS : b); ++m)
                        acc0 = fma(Ab[r0 * b + m], Tb[c0 * b + m], acc0);
                }
                if (e1 < bb) {
#pragma unroll
                    for (int m = 0; m < (BS ? BS : b); ++m)
                        acc1 = fma(Ab[r1 * b + m], Tb[c1 * b + m], acc1);
                }
            }
        }
        int dpos = -1;
        if (D.rp) dpos = find_col(D.ci, D.rp[i], D.rp[i + 1], j);
        if (e0 < bb) {
            double v = alpha * acc0;
            if (dpos >= 0) v = fma(beta, D.v[int64_t(dpos) * bb + e0], v);
            if (i == j && r0 == c0) v += gamma;
            cv[e * bb + e0] = v;
        }
        if (e1 < bb) {
            double v = alpha * acc1;
            if (dpos >= 0) v = fma(beta, D.v[int64_t(dpos) * bb + e1], v);
            if (i == j && r1 == c1) v += gamma;
            cv[e * bb + e1] = v;
        }
    }
}

// Finished values (symmetrised when sym: (C_ij + C_ji^T) / 2) into out, and
// keep[e] = ||block||_F >= sptol.  Warp per block.
__global__ void __launch_bounds__(256) drop_marks(int64_t nnz, int b, const int32_t* row_of,
                                                  const int32_t* rp, const int32_t* ci,
                                                  const double* cv, int sym, double sptol,
                                                  double* out, uint8_t* keep) {
    const int bb = b * b;
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t e = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; e < nnz; e += warps) {
        const int i = row_of[e], j = ci[e];
        const int et = sym ? find_col(ci, rp[j], rp[j + 1], i) : -1;
        double s2 = 0.0;
        for (int el = lane; el < bb; el += 32) {
            double v = cv[e * bb + el];
            if (sym) {
                const int r = el / b, c = el % b;
                v = 0.5 * (v + (et >= 0 ? cv[int64_t(et) * bb + c * b + r] : 0.0));
            }
            out[e * bb + el] = v;
            s2 = fma(v, v, s2);
        }
        for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        if (lane == 0) keep[e] = sqrt(s2) >= sptol ? 1 : 0;
    }
}

// Warp per row: new position of each kept block within its row, row counts.
__global__ void __launch_bounds__(256) keep_positions(int n_rows, const int32_t* rp,
                                                      const uint8_t* keep, int32_t* newpos,
                                                      int32_t* counts) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n_rows; i += warps) {
        int cnt = 0;
        for (int base = rp[i]; base < rp[i + 1]; base += 32) {
            const int e = base + lane;
            const bool k = e < rp[i + 1] && keep[e];
            const unsigned m = __ballot_sync(0xffffffffu, k);
            if (e < rp[i + 1]) newpos[e] = k ? cnt + __popc(m & ((1u << lane) - 1u)) : -1;
            cnt += __popc(m);
        }
        if (lane == 0) counts[i] = cnt;
    }
}

__global__ void compact_copy(int64_t nnz, int b, const int32_t* row_of, const int32_t* ci,
                             const double* vals, const int32_t* newpos, const int32_t* rp_new,
                             int32_t* ci_new, double* v_new) {
    const int64_t bb = int64_t(b) * b;
    const int64_t total = nnz * bb;
    for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < total;
         x += int64_t(gridDim.x) * blockDim.x) {
        const int64_t e = x / bb;
        const int np = newpos[e];
        if (np < 0) continue;
        const int64_t dst = int64_t(rp_new[row_of[e]]) + np;
        const int64_t el = x - e * bb;
        v_new[dst * bb + el] = vals[x];
        if (el == 0) ci_new[dst] = ci[e];
    }
}

// Max over blocks of ||(X - I)[i, j]||_F; a row without a stored diagonal
// block contributes ||-I||_F = sqrt(b) (isqrtm.hpp:360-405).  Warp per row;
// the non-negative doubles are ordered like their bit patterns.
__global__ void __launch_bounds__(256) max_block_residual(int n_rows, int b, const int32_t* rp,
                                                          const int32_t* ci, const double* v,
                                                          unsigned long long* out) {
    const int bb = b * b;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n_rows; i += warps) {
        double worst = 0.0;
        bool diag = false;
        for (int e = rp[i]; e < rp[i + 1]; ++e) {
            const bool d = ci[e] == i;
            diag |= d;
            double s2 = 0.0;
            for (int el = lane; el < bb; el += 32) {
                double x = v[int64_t(e) * bb + el];
                if (d && el / b == el % b) x -= 1.0;
                s2 = fma(x, x, s2);
            }
            for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            worst = fmax(worst, sqrt(s2));
        }
        if (!diag) worst = fmax(worst, sqrt(double(b)));
        if (lane == 0) atomicMax(out, __double_as_longlong(worst));
    }
}

// Block products of A B: sum over A's blocks (., k) of |B row k|.
__global__ void count_products(int64_t nnz_a, const int32_t* aci, const int32_t* brp,
                               unsigned long long* out) {
    unsigned long long s = 0;
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz_a;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int k = aci[p];
        s += unsigned(brp[k + 1] - brp[k]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void sub_inplace(int64_t n, double* y, const double* x) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n;
         t += int64_t(gridDim.x) * blockDim.x)
        y[t] -= x[t];
}

// ------------------------------------------------------------- host side

Pattern pattern_of(const rsatb_bsr_matrix* M) { return {M->row_ptr, M->col_ind}; }
Vals vals_of(const rsatb_bsr_matrix* M) {
    return {M->row_ptr, M->col_ind, static_cast<const double*>(M->values)};
}

enum DropMode { DROP_NONE = 0, DROP_PLAIN = 1, DROP_SYMMETRIC = 2 };

int launch_check(rsatb_context* ctx) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "sparse refinement kernel: %s", cudaGetErrorString(e));
    ctx->launches++;
    return RSATB_SUCCESS;
}

// Host exclusive sum of n device counts into a device row pointer; *total
// receives the sum.
int offsets_from_counts(rsatb_context* ctx, const int32_t* d_counts, int n, int32_t* d_rp,
                        int64_t* total) {
    std::vector<int32_t> c(static_cast<size_t>(n));
    std::vector<int32_t> rp(static_cast<size_t>(n) + 1);
    if (n)
        RSATB_CUDA_TRY(cudaMemcpyAsync(c.data(), d_counts, sizeof(int32_t) * n,
                                       cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    int64_t s = 0;
    for (int i = 0; i < n; ++i) {
        rp[i] = int32_t(s);
        s += c[i];
        if (s > INT32_MAX)
            return set_error(RSATB_OUT_OF_MEMORY, "sparse product exceeds 2^31 blocks");
    }
    rp[n] = int32_t(s);
    RSATB_CUDA_TRY(cudaMemcpyAsync(d_rp, rp.data(), sizeof(int32_t) * (size_t(n) + 1),
                                   cudaMemcpyHostToDevice, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *total = s;
    return RSATB_SUCCESS;
}

// C = alpha A B + beta D + gamma I (D, diagonal optional), BT the transpose
// of B (B itself when B is symmetric), then the sptol drop.
int spgemm(rsatb_context* ctx, const rsatb_bsr_matrix* A, const rsatb_bsr_matrix* B,
           const rsatb_bsr_matrix* BT, const rsatb_bsr_matrix* D, double alpha, double beta,
           double gamma, bool diag, int drop, double sptol, Mat* out) {
    const int n = A->n_block_rows, nbc = B->n_block_cols, b = A->block_size;
    if (A->n_block_cols != B->n_block_rows || BT->n_block_rows != nbc ||
        BT->n_block_cols != B->n_block_rows || B->block_size != b || BT->block_size != b ||
        (D && (D->n_block_rows != n || D->n_block_cols != nbc || D->block_size != b)))
        return set_error(RSATB_INVALID_ARGUMENT, "sparse product: operand shapes differ");
    if ((diag && n != nbc) || b > 8)
        return set_error(RSATB_INVALID_ARGUMENT, "sparse product: bad diagonal term or block size");
    const int words = (nbc + 31) / 32;
    const size_t smem = size_t(words) * sizeof(unsigned);
    if (smem > kMaxBitmapBytes)
        return set_error(RSATB_NOT_SUPPORTED,
                         "sparse product: %d block columns exceed the %zu-byte row bitmap", nbc,
                         kMaxBitmapBytes);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(sym_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kMaxBitmapBytes));
        cudaFuncSetAttribute(sym_fill, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kMaxBitmapBytes));
        attr = true;
    }
    const Pattern pd = D ? pattern_of(D) : Pattern{nullptr, nullptr};
    DevBuf counts;
    RSATB_TRY(dev_alloc(counts, sizeof(int32_t) * (size_t(n) + 1)));
    const int grid_rows = grid_cap(ctx, n, 1);
    sym_count<<<grid_rows, kRowThreads, smem, ctx->stream>>>(n, words, pattern_of(A),
                                                              pattern_of(B), pd, diag ? 1 : 0,
                                                              counts.as<int32_t>());
    RSATB_TRY(launch_check(ctx));
    rsatb_bsr_matrix* raw = nullptr;
    DevBuf rp_tmp;
    RSATB_TRY(dev_alloc(rp_tmp, sizeof(int32_t) * (size_t(n) + 1)));
    int64_t nnz = 0;
    RSATB_TRY(offsets_from_counts(ctx, counts.as<int32_t>(), n, rp_tmp.as<int32_t>(), &nnz));
    RSATB_TRY(alloc_matrix(ctx->device, n, nbc, b, nnz, RSATB_F64, 0, &raw));
    Mat C(raw);
    RSATB_CUDA_TRY(cudaMemcpyAsync(C->row_ptr, rp_tmp.p, sizeof(int32_t) * (size_t(n) + 1),
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    sym_fill<<<grid_rows, kRowThreads, smem, ctx->stream>>>(n, words, pattern_of(A),
                                                             pattern_of(B), pd, diag ? 1 : 0,
                                                             C->row_ptr, C->col_ind);
    RSATB_TRY(launch_check(ctx));
    DevBuf row_of;
    RSATB_TRY(dev_alloc(row_of, sizeof(int32_t) * size_t(std::max<int64_t>(nnz, 1))));
    rows_of_blocks<<<grid_cap(ctx, n, 256), 256, 0, ctx->stream>>>(n, C->row_ptr,
                                                                    row_of.as<int32_t>());
    RSATB_TRY(launch_check(ctx));
    const Vals dv = D ? vals_of(D) : Vals{nullptr, nullptr, nullptr};
    const int grid_blocks = grid_cap(ctx, nnz, 8);
    double* cv = static_cast<double*>(C->values);
    if (nnz) {
        if (b == 8)
            spgemm_numeric<8><<<grid_blocks, 256, 0, ctx->stream>>>(
                nnz, b, row_of.as<int32_t>(), C->col_ind, cv, vals_of(A), vals_of(BT), dv, alpha,
                beta, gamma);
        else
            spgemm_numeric<0><<<grid_blocks, 256, 0, ctx->stream>>>(
                nnz, b, row_of.as<int32_t>(), C->col_ind, cv, vals_of(A), vals_of(BT), dv, alpha,
                beta, gamma);
        RSATB_TRY(launch_check(ctx));
    }
    if (drop == DROP_NONE || nnz == 0) {
        RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        *out = std::move(C);
        return RSATB_SUCCESS;
    }
    const int64_t bb = int64_t(b) * b;
    DevBuf fin, keep, newpos;
    RSATB_TRY(dev_alloc(fin, sizeof(double) * size_t(nnz * bb)));
    RSATB_TRY(dev_alloc(keep, size_t(nnz)));
    RSATB_TRY(dev_alloc(newpos, sizeof(int32_t) * size_t(nnz)));
    drop_marks<<<grid_blocks, 256, 0, ctx->stream>>>(nnz, b, row_of.as<int32_t>(), C->row_ptr,
                                                     C->col_ind, cv, drop == DROP_SYMMETRIC,
                                                     sptol, fin.as<double>(), keep.as<uint8_t>());
    RSATB_TRY(launch_check(ctx));
    keep_positions<<<grid_cap(ctx, n, 8), 256, 0, ctx->stream>>>(
        n, C->row_ptr, keep.as<uint8_t>(), newpos.as<int32_t>(), counts.as<int32_t>());
    RSATB_TRY(launch_check(ctx));
    int64_t kept = 0;
    RSATB_TRY(offsets_from_counts(ctx, counts.as<int32_t>(), n, rp_tmp.as<int32_t>(), &kept));
    rsatb_bsr_matrix* raw2 = nullptr;
    RSATB_TRY(alloc_matrix(ctx->device, n, nbc, b, kept, RSATB_F64, 0, &raw2));
    Mat K(raw2);
    RSATB_CUDA_TRY(cudaMemcpyAsync(K->row_ptr, rp_tmp.p, sizeof(int32_t) * (size_t(n) + 1),
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    compact_copy<<<grid_cap(ctx, nnz * bb, 256), 256, 0, ctx->stream>>>(
        nnz, b, row_of.as<int32_t>(), C->col_ind, fin.as<double>(), newpos.as<int32_t>(),
        K->row_ptr, K->col_ind, static_cast<double*>(K->values));
    RSATB_TRY(launch_check(ctx));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *out = std::move(K);
    return RSATB_SUCCESS;
}

int transpose(rsatb_context* ctx, const rsatb_bsr_matrix* A, Mat* out) {
    rsatb_bsr_t t = nullptr;
    RSATB_TRY(rsatb_bsr_adjoint(ctx, const_cast<rsatb_bsr_matrix*>(A), &t));
    out->reset(t);
    return RSATB_SUCCESS;
}

int residual_of(rsatb_context* ctx, const rsatb_bsr_matrix* X, double* out) {
    DevBuf d;
    RSATB_TRY(dev_alloc(d, sizeof(unsigned long long)));
    RSATB_CUDA_TRY(cudaMemsetAsync(d.p, 0, sizeof(unsigned long long), ctx->stream));
    max_block_residual<<<grid_cap(ctx, X->n_block_rows, 8), 256, 0, ctx->stream>>>(
        X->n_block_rows, X->block_size, X->row_ptr, X->col_ind,
        static_cast<const double*>(X->values), d.as<unsigned long long>());
    RSATB_TRY(launch_check(ctx));
    unsigned long long h = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(&h, d.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, &h, sizeof(double));
    return RSATB_SUCCESS;
}

int products(rsatb_context* ctx, const rsatb_bsr_matrix* A, const rsatb_bsr_matrix* B,
             double* out) {
    DevBuf d;
    RSATB_TRY(dev_alloc(d, sizeof(unsigned long long)));
    RSATB_CUDA_TRY(cudaMemsetAsync(d.p, 0, sizeof(unsigned long long), ctx->stream));
    if (A->nnz_blocks) {
        count_products<<<grid_cap(ctx, A->nnz_blocks, 256), 256, 0, ctx->stream>>>(
            A->nnz_blocks, A->col_ind, B->row_ptr, d.as<unsigned long long>());
        RSATB_TRY(launch_check(ctx));
    }
    unsigned long long h = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(&h, d.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *out = double(h);
    return RSATB_SUCCESS;
}

int copy_matrix(rsatb_context* ctx, const rsatb_bsr_matrix* A, Mat* out) {
    rsatb_bsr_matrix* raw = nullptr;
    RSATB_TRY(alloc_matrix(ctx->device, A->n_block_rows, A->n_block_cols, A->block_size,
                           A->nnz_blocks, RSATB_F64, 0, &raw));
    Mat C(raw);
    const size_t bb = size_t(A->block_size) * A->block_size;
    RSATB_CUDA_TRY(cudaMemcpyAsync(C->row_ptr, A->row_ptr,
                                   sizeof(int32_t) * (size_t(A->n_block_rows) + 1),
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    if (A->nnz_blocks) {
        RSATB_CUDA_TRY(cudaMemcpyAsync(C->col_ind, A->col_ind,
                                       sizeof(int32_t) * size_t(A->nnz_blocks),
                                       cudaMemcpyDeviceToDevice, ctx->stream));
        RSATB_CUDA_TRY(cudaMemcpyAsync(C->values, A->values,
                                       sizeof(double) * size_t(A->nnz_blocks) * bb,
                                       cudaMemcpyDeviceToDevice, ctx->stream));
    }
    *out = std::move(C);
    return RSATB_SUCCESS;
}

// ||(Z^H S Z - I) v|| for v a unit random vector (seed 1), through the
// fused step kernels (isqrtm.hpp:324-339).
int applied_residual(rsatb_context* ctx, const rsatb_bsr_matrix* S, const rsatb_bsr_matrix* Z,
                     const rsatb_bsr_matrix* ZT, double* out) {
    const int64_t n = int64_t(S->n_block_rows) * S->block_size;
    DevBuf v, w, u, y;
    RSATB_TRY(dev_alloc(v, sizeof(double) * n));
    RSATB_TRY(dev_alloc(w, sizeof(double) * n));
    RSATB_TRY(dev_alloc(u, sizeof(double) * n));
    RSATB_TRY(dev_alloc(y, sizeof(double) * n));
    std::vector<int64_t> ids(static_cast<size_t>(S->n_block_rows));
    for (size_t a = 0; a < ids.size(); ++a) ids[a] = int64_t(a);
    RSATB_TRY(rsatb_set_random(ctx, 1, RSATB_RANDOM_UNIFORM, 1, ids.data(), int(ids.size()),
                               S->block_size, n, 1, 0, RSATB_F64, v.p));
    auto apply = [&](const rsatb_bsr_matrix* A, const void* x, void* yy) {
        StepArgs a{};
        a.W = 1;
        a.in = x;
        a.y = yy;
        a.s_in = 1.0;
        a.s_out = 1.0;
        a.s2 = 1.0;
        a.dot_mode = DOT_NONE;
        return run_step(ctx, A, RSATB_F64, a);
    };
    RSATB_TRY(apply(Z, v.p, w.p));
    RSATB_TRY(apply(S, w.p, u.p));
    RSATB_TRY(apply(ZT, u.p, y.p));
    sub_inplace<<<grid_cap(ctx, n, 256), 256, 0, ctx->stream>>>(n, y.as<double>(),
                                                               v.as<double>());
    RSATB_TRY(launch_check(ctx));
    std::vector<double> hv(static_cast<size_t>(n)), hy(static_cast<size_t>(n));
    RSATB_CUDA_TRY(cudaMemcpyAsync(hv.data(), v.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(hy.data(), y.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RSATB_TRY(ctx_check_fault(ctx));
    double nv = 0.0, ny = 0.0;
    for (int64_t t = 0; t < n; ++t) {
        nv += hv[t] * hv[t];
        ny += hy[t] * hy[t];
    }
    *out = nv > 0.0 ? std::sqrt(ny / nv) : 0.0;
    return RSATB_SUCCESS;
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_inverse_sqrt_refine(rsatb_ctx_t ctx, rsatb_bsr_t S, rsatb_bsr_t Z_seed,
                                         const rsatb_ns_refine_options* options,
                                         rsatb_bsr_t* Z_out, rsatb_ns_refine_report* report) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_TRY(check_bsr(S, "S"));
    RSATB_TRY(check_bsr(Z_seed, "Z_seed"));
    if (!options || !Z_out) return set_error(RSATB_INVALID_ARGUMENT, "null options or output");
    *Z_out = nullptr;
    if (S->dtype != RSATB_F64 || Z_seed->dtype != RSATB_F64 || (S->flags | Z_seed->flags))
        return set_error(RSATB_NOT_SUPPORTED,
                         "the sparse refinement takes real FP64 S and seed (complex overlaps "
                         "are not served)");
    if (S->n_block_rows != S->n_block_cols || Z_seed->n_block_rows != S->n_block_rows ||
        Z_seed->n_block_cols != S->n_block_cols || Z_seed->block_size != S->block_size)
        return set_error(RSATB_INVALID_ARGUMENT, "S must be square and the seed of its shape");
    if (S->block_size > 8)
        return set_error(RSATB_NOT_SUPPORTED,
                         "blocks above 8 x 8 are not served (a warp holds 64 block elements)");
    const double tol = options->tol, sptol = options->sptol;
    const int maxit = options->maxit;
    if (!(tol >= 0.0) || !(sptol >= 0.0) || maxit < 0)
        return set_error(RSATB_INVALID_ARGUMENT, "tol, sptol and maxit must be non-negative");

    rsatb_ns_refine_report rep{};
    Mat Z, ZT, X, P, U, UT, T;
    RSATB_TRY(copy_matrix(ctx, Z_seed, &Z));
    RSATB_TRY(transpose(ctx, Z.get(), &ZT));

    auto reform = [&]() -> int {
        // X = Z^H S Z: U = S Z, then Z^H U with U^T = (S Z)^T, symmetrised.
        RSATB_TRY(spgemm(ctx, S, Z.get(), ZT.get(), nullptr, 1.0, 0.0, 0.0, false, DROP_NONE,
                         0.0, &U));
        RSATB_TRY(transpose(ctx, U.get(), &UT));
        RSATB_TRY(spgemm(ctx, ZT.get(), U.get(), UT.get(), nullptr, 1.0, 0.0, 0.0, false,
                         DROP_SYMMETRIC, sptol, &X));
        U.reset();
        UT.reset();
        rep.reforms++;
        return RSATB_SUCCESS;
    };

    if (maxit > 0) {
        RSATB_TRY(reform());
        double norm = 0.0, norm_pre = 0.0;
        RSATB_TRY(residual_of(ctx, X.get(), &norm));
        int count = 0;
        while (norm > tol && count < maxit && std::fabs(norm_pre - norm) > 0.005 * norm) {
            if (norm > 100.0) {
                rep.diverged = 1;
                break;
            }
            norm_pre = norm;
            // P = 0.375 X^2 - 1.25 X + 1.875 I (X symmetric: X^T = X).
            RSATB_TRY(spgemm(ctx, X.get(), X.get(), X.get(), X.get(), 0.375, -1.25, 1.875, true,
                             DROP_SYMMETRIC, sptol, &P));
            // Z <- Z P (P symmetric).
            Mat Zn;
            RSATB_TRY(spgemm(ctx, Z.get(), P.get(), P.get(), nullptr, 1.0, 0.0, 0.0, false,
                             DROP_PLAIN, sptol, &Zn));
            Z = std::move(Zn);
            RSATB_TRY(transpose(ctx, Z.get(), &ZT));
            // Route: propagation X <- P X P contracts X but drifts; every
            // fifth step, and while the residual is 0.1 or above, X is
            // reformed exactly (isqrtm.hpp:712-745).  Otherwise the route
            // with fewer block products in its first product wins.
            bool propagate = false;
            if (options->route == 0 && (count + 1) % 5 != 0 && norm < 1e-1) {
                double pr = 0.0, pp = 0.0;
                RSATB_TRY(products(ctx, S, Z.get(), &pr));
                RSATB_TRY(products(ctx, P.get(), X.get(), &pp));
                propagate = pp < pr;
            }
            if (propagate) {
                RSATB_TRY(spgemm(ctx, P.get(), X.get(), X.get(), nullptr, 1.0, 0.0, 0.0, false,
                                 DROP_NONE, 0.0, &T));
                RSATB_TRY(spgemm(ctx, T.get(), P.get(), P.get(), nullptr, 1.0, 0.0, 0.0, false,
                                 DROP_SYMMETRIC, sptol, &X));
                T.reset();
                rep.propagations++;
            } else {
                X.reset();
                RSATB_TRY(reform());
            }
            P.reset();
            RSATB_TRY(residual_of(ctx, X.get(), &norm));
            ++count;
            rep.last_advance_propagated = propagate ? 1 : 0;
        }
        rep.steps = count;
        rep.residual = norm;
        rep.converged = norm <= tol ? 1 : 0;
        rep.hit_maxiter = count >= maxit ? 1 : 0;
    }
    RSATB_TRY(applied_residual(ctx, S, Z.get(), ZT.get(), &rep.applied_residual));
    rep.nnz_blocks = Z->nnz_blocks;
    if (report) *report = rep;
    *Z_out = Z.release();
    return RSATB_SUCCESS;
}
