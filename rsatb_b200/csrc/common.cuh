// Shared host/device definitions of the rsatb_b200 library: the handle
// structs behind the C ABI, error plumbing and scalar traits.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <string>

#include "../../include/rsatb_b200.h"

namespace rsatb_b200 {

// ---------------------------------------------------------------- errors

// Records `msg` as the calling thread's last error and returns `status`.
int set_error(int status, const char* fmt, ...);
void clear_error();

#define RSATB_CUDA_TRY(call)                                                     \
    do {                                                                        \
        cudaError_t err_ = (call);                                              \
        if (err_ != cudaSuccess) {                                              \
            return ::rsatb_b200::set_error(                                     \
                err_ == cudaErrorMemoryAllocation ? RSATB_OUT_OF_MEMORY          \
                                                  : RSATB_CUDA_ERROR,            \
                "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_),       \
                __FILE__, __LINE__);                                            \
        }                                                                       \
    } while (0)

// Checks the launch just issued on the current thread.
#define RSATB_LAUNCH_CHECK(ctx)                                                  \
    do {                                                                        \
        cudaError_t err_ = cudaGetLastError();                                  \
        if (err_ != cudaSuccess) {                                              \
            return ::rsatb_b200::set_error(RSATB_CUDA_ERROR,                    \
                "kernel launch failed: %s (%s:%d)", cudaGetErrorString(err_),    \
                __FILE__, __LINE__);                                            \
        }                                                                       \
        (ctx)->launches++;                                                      \
    } while (0)

#define RSATB_TRY(expr)                  \
    do {                                \
        int st_ = (expr);               \
        if (st_ != RSATB_SUCCESS) return st_; \
    } while (0)

// --------------------------------------------------------------- handles

}  // namespace rsatb_b200

struct rsatb_context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // Grow-only device scratch (partial dot sums, sandwich intermediates);
    // released with the context.
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // Completion counters of the last-block reductions, zero between launches.
    unsigned* counters = nullptr;
    int n_counters = 0;
    int64_t launches = 0;
    // The KPM moment recurrence as a captured CUDA graph, replayed while the
    // call's arguments (key) are unchanged; the key of the last direct run
    // decides when to capture (the second identical call).
    cudaGraphExec_t kpm_graph = nullptr;
    std::string kpm_graph_key;
    std::string kpm_seen_key;
    int64_t kpm_graph_launches = 0;
    // Pinned host staging (grow-only) for small asynchronous read-backs.
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
};

struct rsatb_bsr_matrix {
    int device = 0;
    int n_block_rows = 0;
    int n_block_cols = 0;
    int block_size = 0;
    int64_t nnz_blocks = 0;
    int32_t* row_ptr = nullptr;   // device
    int32_t* col_ind = nullptr;   // device
    void* values = nullptr;       // device
    int dtype = RSATB_F64;
    unsigned flags = 0;           // only RSATB_BSR_IMAGINARY_UNIT is kept
    int max_row_blocks = 0;
};

namespace rsatb_b200 {

inline bool dtype_is_complex(int t) { return t == RSATB_C128 || t == RSATB_C64; }
inline bool dtype_is_double(int t) { return t == RSATB_F64 || t == RSATB_C128; }
inline bool dtype_valid(int t) { return t >= RSATB_F64 && t <= RSATB_C64; }
inline size_t dtype_size(int t) {
    switch (t) {
        case RSATB_F64: return 8;
        case RSATB_F32: return 4;
        case RSATB_C128: return 16;
        case RSATB_C64: return 8;
    }
    return 0;
}
// Size of the real component type (8 for F64/C128, 4 for F32/C64).
inline size_t dtype_real_size(int t) { return dtype_is_double(t) ? 8 : 4; }

// Scratch of at least `bytes`, 256-byte aligned; grows (synchronising the
// stream) when too small.  Valid until the next call that grows it.
int ctx_scratch(rsatb_context* ctx, size_t bytes, void** out);
// Pointer to `n` zeroed completion counters.
int ctx_counters(rsatb_context* ctx, int n, unsigned** out);
// The context's device fault word (the last of its 64 counters): kernels
// whose bounded waits give up set it non-zero.
int ctx_fault_word(rsatb_context* ctx, unsigned** out);
// Pinned host memory of at least `bytes` (grow-only, released with the
// context).
int ctx_pinned(rsatb_context* ctx, size_t bytes, void** out);
// After the stream has been synchronised: reads and clears the fault word;
// RSATB_CUDA_ERROR when a kernel recorded a fault.
int ctx_check_fault(rsatb_context* ctx);

int check_ctx(rsatb_context* ctx);
int check_bsr(const rsatb_bsr_matrix* A, const char* name);

// A matrix shell with device arrays for nnzb blocks (row_ptr, col_ind and
// values left unset), and its release.
int alloc_matrix(int device, int nbr, int nbc, int b, int64_t nnzb, int dtype, unsigned flags,
                 rsatb_bsr_matrix** out);
void free_matrix(rsatb_bsr_matrix* A);

}  // namespace rsatb_b200
