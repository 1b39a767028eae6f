// Context, memory and error entry points of the C ABI.
#include "common.cuh"

#include <mutex>
#include <vector>

namespace rsatb_b200 {

namespace {
thread_local std::string g_last_error;
}

int set_error(int status, const char* fmt, ...) {
    char buf[1024];
    va_list args;
    va_start(args, fmt);
    vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    g_last_error = buf;
    return status;
}

void clear_error() { g_last_error.clear(); }

int check_ctx(rsatb_context* ctx) {
    if (ctx == nullptr) return set_error(RSATB_INVALID_ARGUMENT, "null context");
    cudaError_t err = cudaSetDevice(ctx->device);
    if (err != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "cudaSetDevice(%d): %s", ctx->device,
                         cudaGetErrorString(err));
    return RSATB_SUCCESS;
}

int check_bsr(const rsatb_bsr_matrix* A, const char* name) {
    if (A == nullptr) return set_error(RSATB_INVALID_ARGUMENT, "%s: null matrix", name);
    if (A->n_block_rows < 0 || A->block_size <= 0)
        return set_error(RSATB_INVALID_ARGUMENT, "%s: malformed matrix", name);
    return RSATB_SUCCESS;
}

int ctx_scratch(rsatb_context* ctx, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    if (ctx->scratch_bytes < bytes) {
        if (ctx->scratch) {
            RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            RSATB_CUDA_TRY(cudaFree(ctx->scratch));
            ctx->scratch = nullptr;
            ctx->scratch_bytes = 0;
        }
        // Grow geometrically so that a sequence of slightly larger requests
        // does not reallocate every time.
        size_t grow = bytes + bytes / 4;
        RSATB_CUDA_TRY(cudaMalloc(&ctx->scratch, grow));
        ctx->scratch_bytes = grow;
    }
    *out = ctx->scratch;
    return RSATB_SUCCESS;
}

int ctx_counters(rsatb_context* ctx, int n, unsigned** out) {
    if (ctx->n_counters < n) {
        if (ctx->counters) {
            RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            RSATB_CUDA_TRY(cudaFree(ctx->counters));
            ctx->counters = nullptr;
        }
        int m = n < 64 ? 64 : n + 1;
        RSATB_CUDA_TRY(cudaMalloc(&ctx->counters, sizeof(unsigned) * m));
        RSATB_CUDA_TRY(cudaMemsetAsync(ctx->counters, 0, sizeof(unsigned) * m, ctx->stream));
        ctx->n_counters = m;
    }
    *out = ctx->counters;
    return RSATB_SUCCESS;
}

int ctx_pinned(rsatb_context* ctx, size_t bytes, void** out) {
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) {
            RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            RSATB_CUDA_TRY(cudaFreeHost(ctx->pinned));
            ctx->pinned = nullptr;
            ctx->pinned_bytes = 0;
        }
        const size_t grow = bytes < 4096 ? 4096 : bytes + bytes / 2;
        RSATB_CUDA_TRY(cudaHostAlloc(&ctx->pinned, grow, cudaHostAllocDefault));
        ctx->pinned_bytes = grow;
    }
    *out = ctx->pinned;
    return RSATB_SUCCESS;
}

int ctx_fault_word(rsatb_context* ctx, unsigned** out) {
    unsigned* c = nullptr;
    RSATB_TRY(ctx_counters(ctx, 1, &c));
    *out = c + (ctx->n_counters - 1);
    return RSATB_SUCCESS;
}

int ctx_check_fault(rsatb_context* ctx) {
    if (!ctx->counters) return RSATB_SUCCESS;
    unsigned* w = ctx->counters + (ctx->n_counters - 1);
    unsigned h = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h == 0) return RSATB_SUCCESS;
    RSATB_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(unsigned), ctx->stream));
    return set_error(RSATB_CUDA_ERROR,
                     "a step kernel gave up waiting for its bulk copies (bounded wait), in this "
                     "call or in an earlier asynchronous call on this context");
}

}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" {

const char* rsatb_last_error(void) { return g_last_error.c_str(); }

int rsatb_version(void) { return 100; }

int rsatb_ctx_create(int device, rsatb_ctx_t* out) {
    clear_error();
    if (out == nullptr) return set_error(RSATB_INVALID_ARGUMENT, "null output pointer");
    int n_dev = 0;
    RSATB_CUDA_TRY(cudaGetDeviceCount(&n_dev));
    if (device < 0 || device >= n_dev)
        return set_error(RSATB_INVALID_ARGUMENT, "device %d out of range (%d devices)", device,
                         n_dev);
    RSATB_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    RSATB_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return set_error(RSATB_NOT_SUPPORTED,
                         "device %d is sm_%d%d; this library is built for sm_100a only", device,
                         prop.major, prop.minor);
    auto* ctx = new rsatb_context();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    cudaError_t err = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete ctx;
        return set_error(RSATB_CUDA_ERROR, "cudaStreamCreate: %s", cudaGetErrorString(err));
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return RSATB_SUCCESS;
}

int rsatb_ctx_destroy(rsatb_ctx_t ctx) {
    clear_error();
    if (ctx == nullptr) return RSATB_SUCCESS;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->counters) cudaFree(ctx->counters);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->kpm_graph) cudaGraphExecDestroy(ctx->kpm_graph);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return RSATB_SUCCESS;
}

int rsatb_ctx_set_stream(rsatb_ctx_t ctx, void* stream) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    // Work already queued on the old stream must precede work on the new one.
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->stream = static_cast<cudaStream_t>(stream);
    return RSATB_SUCCESS;
}

void* rsatb_ctx_stream(rsatb_ctx_t ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int rsatb_ctx_synchronize(rsatb_ctx_t ctx) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    // Bounded waits that gave up in asynchronous calls queued on this context
    // (mult_dense, apply_op, apply_dual, propagate) are reported here.
    return ctx_check_fault(ctx);
}

int64_t rsatb_ctx_launch_count(rsatb_ctx_t ctx) { return ctx ? ctx->launches : 0; }

int rsatb_device_alloc(rsatb_ctx_t ctx, size_t bytes, void** out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (out == nullptr) return set_error(RSATB_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    if (bytes == 0) return RSATB_SUCCESS;
    RSATB_CUDA_TRY(cudaMalloc(out, bytes));
    return RSATB_SUCCESS;
}

int rsatb_device_free(rsatb_ctx_t ctx, void* ptr) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (ptr == nullptr) return RSATB_SUCCESS;
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RSATB_CUDA_TRY(cudaFree(ptr));
    return RSATB_SUCCESS;
}

int rsatb_copy_to_device(rsatb_ctx_t ctx, void* dst, const void* src, size_t bytes) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (bytes == 0) return RSATB_SUCCESS;
    if (!dst || !src) return set_error(RSATB_INVALID_ARGUMENT, "null pointer in copy");
    RSATB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    return RSATB_SUCCESS;
}

int rsatb_copy_to_host_sync(rsatb_ctx_t ctx, void* dst, const void* src, size_t bytes) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (bytes == 0) return RSATB_SUCCESS;
    if (!dst || !src) return set_error(RSATB_INVALID_ARGUMENT, "null pointer in copy");
    RSATB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return RSATB_SUCCESS;
}

}  // extern "C"
