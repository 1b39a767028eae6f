// rsatb_kpm_dos_moments_noalloc: the KPM moment recurrence of
// rsatb_kpm_dos_moments with no device allocation at all.
//
// Who needs it: callers that cannot (or must not) call cudaMalloc.  Two
// common cases are a process whose device memory is already reserved in
// full by another allocator -- a framework's caching pool sized to the whole
// GPU -- where a fresh cudaMalloc fails or fragments that pool, and a
// latency-sensitive loop that cannot accept the implicit device-wide
// synchronisation of cudaMalloc/cudaFree.  Such callers pass inputs and
// outputs they own; every temporary of the recurrence (the three rotating
// panels, the sandwich intermediates, the per-CTA dot partials, the per-step
// dots and the completion counter) lives in one file-scope device array of
// kNoAllocScratchBytes (32 MiB).  Each GPU that loads the library holds that
// array until the process exits.
//
// The array's name is only a host-side stand-in in host code; its device
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call on that device, so that first call does
// the set-up and should come before any stream capture.  All calls share the
// array and it keeps the last call's contents: the array's 256-byte header
// (the completion counter of the dot reductions and the fault word of the
// step kernels' bounded waits) is cleared at the start of every call,
// everything else is written before it is read.  The fault word lives in
// the header, not in the context, so that no context counter is ever
// allocated on this path; it is read back with the dots, and a wait that
// gave up fails the call with RSATB_CUDA_ERROR.  Calls that overlap on the
// GPU (two streams, two host threads) race on the array; serialise them.
//
// With lazy module loading (the default since CUDA 12.2) the array is
// reserved when this file's module is loaded, which the first call's
// cudaGetSymbolAddress does: on a device whose memory another allocator
// will take in full, make the first call (for example on a tiny problem)
// before that allocator reserves the device.
#include "cheb_kernels.cuh"

#include <cmath>
#include <complex>
#include <mutex>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a);
int run_coldot(rsatb_context* ctx, int vdt, int64_t n_rows, const StepArgs& a);

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (which must be current).
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices)
        return set_error(RSATB_NOT_SUPPORTED, "no-alloc scratch: device %d beyond %d", device,
                         kMaxDevices);
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (g_addr[device] == nullptr) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || p == nullptr)
            return set_error(RSATB_CUDA_ERROR, "cudaGetSymbolAddress(no-alloc scratch): %s",
                             cudaGetErrorString(err));
        g_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_addr[device]);
    return RSATB_SUCCESS;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Step arguments with the fault word of the static array's header, so that
// run_step never falls back to the context's (allocated) fault word.
StepArgs blank(int W, unsigned* fault) {
    StepArgs a{};
    a.W = W;
    a.s_in = 1.0;
    a.s_out = 1.0;
    a.s2 = 1.0;
    a.dot_mode = DOT_NONE;
    a.fault = fault;
    return a;
}

int check_square(const rsatb_bsr_matrix* A, int vdt, const char* name) {
    RSATB_TRY(check_bsr(A, name));
    if (A->n_block_rows != A->n_block_cols)
        return set_error(RSATB_INVALID_ARGUMENT, "%s must be square", name);
    if (!dtype_valid(vdt) || dtype_is_double(A->dtype) != dtype_is_double(vdt))
        return set_error(RSATB_INVALID_ARGUMENT, "%s precision differs from the multivector's",
                         name);
    if (dtype_is_complex(A->dtype) && !dtype_is_complex(vdt))
        return set_error(RSATB_INVALID_ARGUMENT, "%s is complex but the multivector is real",
                         name);
    return RSATB_SUCCESS;
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_kpm_dos_moments_noalloc(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                             const void* psi, int n_vectors,
                                             rsatb_dtype vec_dtype, int n_moments, int doubled,
                                             double* mu_out, double* col_mu_out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!op) return set_error(RSATB_INVALID_ARGUMENT, "null operator");
    RSATB_TRY(check_square(op->H, vec_dtype, "H"));
    const bool sandwich = op->form == RSATB_FORM_SANDWICH;
    if (!sandwich && op->form != RSATB_FORM_ORTHOGONAL)
        return set_error(RSATB_NOT_SUPPORTED, "operator form %d is not available", op->form);
    const int64_t n_rows = int64_t(op->H->n_block_rows) * op->H->block_size;
    if (sandwich) {
        RSATB_TRY(check_square(op->Z, vec_dtype, "Z"));
        RSATB_TRY(check_square(op->ZH, vec_dtype, "ZH"));
        if (int64_t(op->Z->n_block_rows) * op->Z->block_size != n_rows ||
            int64_t(op->ZH->n_block_rows) * op->ZH->block_size != n_rows)
            return set_error(RSATB_INVALID_ARGUMENT, "Z, Z^H and H sizes differ");
    }
    if (!(op->half_width > 0.0) || !std::isfinite(op->half_width) || !std::isfinite(op->center))
        return set_error(RSATB_INVALID_ARGUMENT, "spectral window needs half_width > 0");
    if (n_vectors <= 0 || n_moments <= 0 || !psi || !mu_out)
        return set_error(RSATB_INVALID_ARGUMENT, "bad n_vectors, n_moments, psi or mu_out");
    if (!aligned16(psi)) return set_error(RSATB_INVALID_ARGUMENT, "psi must be 16-byte aligned");
    const bool cv = dtype_is_complex(vec_dtype);
    const int R = n_vectors;
    const int W = R * (cv ? 2 : 1);
    if (W > 1536) return set_error(RSATB_NOT_SUPPORTED, "too many vectors (W = %d > 1536)", W);

    int n_steps = 0;
    if (n_moments > 1) {
        if (doubled) {
            n_steps = 1;
            for (int n = 1; 2 * n + 1 < n_moments; ++n) ++n_steps;
        } else {
            n_steps = n_moments - 1;
        }
    }

    // Carve the static array: counter, panels, sandwich pair, partials, dots.
    const size_t vbytes = round256(size_t(n_rows) * W * dtype_real_size(vec_dtype));
    const size_t max_ctas = size_t(ctx->sm_count) * 8;
    const size_t part_bytes = round256(max_ctas * 2 * W * sizeof(double));
    const size_t dots_bytes = round256(size_t(n_steps + 1) * 2 * W * sizeof(double));
    const int n_panels = 3 + (sandwich ? 2 : 0);
    const size_t need = 256 + n_panels * vbytes + part_bytes + dots_bytes;
    if (need > kNoAllocScratchBytes)
        return set_error(RSATB_INVALID_ARGUMENT,
                         "rsatb_kpm_dos_moments_noalloc: this problem needs %zu bytes of "
                         "scratch, beyond the fixed %zu-byte (32 MiB) static array; use "
                         "rsatb_kpm_dos_moments",
                         need, kNoAllocScratchBytes);
    unsigned char* base = nullptr;
    RSATB_TRY(scratch_address(ctx->device, &base));
    // Header: the dot reductions' completion counter at byte 0, the step
    // kernels' fault word at byte 128.
    unsigned* counter = reinterpret_cast<unsigned*>(base);
    unsigned* fault = reinterpret_cast<unsigned*>(base + 128);
    unsigned char* p = base + 256;
    void* buf[3] = {p, p + vbytes, p + 2 * vbytes};
    void* u = sandwich ? p + 3 * vbytes : nullptr;
    void* w = sandwich ? p + 4 * vbytes : nullptr;
    double* partials = reinterpret_cast<double*>(p + n_panels * vbytes);
    double* dots = reinterpret_cast<double*>(p + n_panels * vbytes + part_bytes);
    // The last-CTA reductions need a zero counter and the fault word starts
    // clear; the previous call left the counter at zero, but a call that
    // failed half-way may not have.
    RSATB_CUDA_TRY(cudaMemsetAsync(base, 0, 256, ctx->stream));

    {
        StepArgs a = blank(W, fault);
        a.x = psi;
        a.in = psi;
        a.partials = partials;
        a.dots_out = dots;
        a.counter = counter;
        RSATB_TRY(run_coldot(ctx, vec_dtype, n_rows, a));
    }
    const double inv_hw = 1.0 / op->half_width;
    const void* prev = nullptr;
    const void* cur = psi;
    int slot = 0;
    for (int s = 1; s <= n_steps; ++s) {
        void* out = buf[slot];
        slot = (slot + 1) % 3;
        StepArgs last = blank(W, fault);
        last.x = cur;
        last.p = (s == 1) ? nullptr : prev;
        last.psi0 = psi;
        last.y = out;
        last.c = op->center;
        last.s_out = inv_hw;
        last.s2 = (s == 1) ? 1.0 : 2.0;
        last.g_p = (s == 1) ? 0.0 : -1.0;
        last.dot_mode = doubled ? DOT_DOUBLING : DOT_PLAIN;
        last.partials = partials;
        last.dots_out = dots + size_t(s) * 2 * W;
        last.counter = counter;
        if (sandwich) {
            StepArgs a = blank(W, fault);
            a.in = cur;
            a.y = u;
            RSATB_TRY(run_step(ctx, op->Z, vec_dtype, a));
            a.in = u;
            a.y = w;
            RSATB_TRY(run_step(ctx, op->H, vec_dtype, a));
            last.in = w;
            RSATB_TRY(run_step(ctx, op->ZH, vec_dtype, last));
        } else {
            last.in = cur;
            RSATB_TRY(run_step(ctx, op->H, vec_dtype, last));
        }
        prev = cur;
        cur = out;
    }

    std::vector<double> h(size_t(n_steps + 1) * 2 * W);
    unsigned fault_h = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), dots, sizeof(double) * h.size(),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(&fault_h, fault, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (fault_h)
        return set_error(RSATB_CUDA_ERROR,
                         "a step kernel gave up waiting for its bulk copies (bounded wait); the "
                         "moments of this call are not valid");

    using cd = std::complex<double>;
    auto coldot = [&](int s, int d, int q) -> cd {
        const double* v = h.data() + size_t(s) * 2 * W + size_t(d) * W;
        return cv ? cd(v[2 * q], v[2 * q + 1]) : cd(v[q], 0.0);
    };
    // Same formulas and column-averaging order as rsatb_kpm_dos_moments
    // (rsatb/calc/dos.hpp:134-173).
    auto avg = [&](auto f) {
        cd s(0.0, 0.0);
        for (int q = 0; q < R; ++q) s += f(q);
        return s / double(R);
    };
    std::vector<cd> mu(n_moments, cd(0.0, 0.0));
    mu[0] = avg([&](int q) { return coldot(0, 0, q); });
    if (n_moments > 1) {
        if (doubled) {
            mu[1] = avg([&](int q) { return std::conj(coldot(1, 0, q)); });
            for (int s = 1; s <= n_steps; ++s) {
                if (2 * s - 1 < n_moments && 2 * s - 1 > 1)
                    mu[2 * s - 1] = 2.0 * avg([&](int q) { return coldot(s, 0, q); }) - mu[1];
                if (2 * s < n_moments)
                    mu[2 * s] = 2.0 * avg([&](int q) { return coldot(s, 1, q); }) - mu[0];
            }
        } else {
            for (int s = 1; s <= n_steps; ++s) mu[s] = avg([&](int q) { return coldot(s, 0, q); });
        }
    }
    for (int n = 0; n < n_moments; ++n) {
        mu_out[2 * n] = mu[n].real();
        mu_out[2 * n + 1] = mu[n].imag();
    }
    if (col_mu_out) {
        for (int q = 0; q < R; ++q) {
            std::vector<cd> c(n_moments, cd(0.0, 0.0));
            c[0] = coldot(0, 0, q);
            if (n_moments > 1) {
                if (doubled) {
                    c[1] = std::conj(coldot(1, 0, q));
                    for (int s = 1; s <= n_steps; ++s) {
                        if (2 * s - 1 < n_moments && 2 * s - 1 > 1)
                            c[2 * s - 1] = 2.0 * coldot(s, 0, q) - c[1];
                        if (2 * s < n_moments) c[2 * s] = 2.0 * coldot(s, 1, q) - c[0];
                    }
                } else {
                    for (int s = 1; s <= n_steps; ++s) c[s] = coldot(s, 0, q);
                }
            }
            for (int n = 0; n < n_moments; ++n) {
                col_mu_out[2 * (size_t(n) * R + q)] = c[n].real();
                col_mu_out[2 * (size_t(n) * R + q) + 1] = c[n].imag();
            }
        }
    }
    return RSATB_SUCCESS;
}
