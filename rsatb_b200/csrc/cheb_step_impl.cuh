// Launch-shape selection and template dispatch of the fused step, included
// once per precision (cheb_step_f64.cu, cheb_step_f32.cu).
#pragma once

#include "cheb_kernels.cuh"
#include "cheb_staged.cuh"
#include "cheb_rowsplit.cuh"
#include "cheb_bulk.cuh"
#include "cheb_narrow.cuh"
#include "cheb_dmma.cuh"
#include "cheb_tf32.cuh"

#include <cstdlib>
#include <mutex>
#include <unordered_map>

namespace rsatb_b200 {
namespace step_detail {

// Resident CTAs per SM for a kernel at a given CTA size and shared memory.
inline int occupancy(const void* kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::unordered_map<uint64_t, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t key = (uint64_t(reinterpret_cast<uintptr_t>(kernel)) << 8) ^
                         (uint64_t(threads) << 40) ^ (uint64_t(smem) << 20) ^ uint64_t(dev);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    int n = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess ||
        n < 1)
        n = 1;
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = n;
    return n;
}

// Optional tuning override of the values-per-thread choice (RSATB_STEP_V).
inline int env_v() {
    const char* s = std::getenv("RSATB_STEP_V");
    return s ? std::atoi(s) : 0;
}

template <typename Kernel>
int launch(rsatb_context* ctx, Kernel kernel, int V, int64_t rows, StepArgs& a) {
    const int L = a.W / V;
    const int threads = L * (256 / L);
    const int ndots = a.dot_mode == DOT_DOUBLING ? 2 : (a.dot_mode == DOT_PLAIN ? 1 : 0);
    const size_t smem = size_t(ndots ? 2 : 0) * threads * V * sizeof(double);
    const int64_t need = (rows * L + threads - 1) / threads;
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, smem);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (grid > int64_t(ctx->sm_count) * 8) grid = int64_t(ctx->sm_count) * 8;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, smem, ctx->stream>>>(a);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

// Picks V (values per thread) for W real values per row.
inline int pick_v(int W, bool cv, bool any_b, int block_size, bool dbl) {
    const int forced = env_v();
    auto ok = [&](int v) {
        if (v <= 0 || W % v) return false;
        if (cv && v % 2) return false;
        return W / v <= 256;
    };
    if (forced && ok(forced) && (!any_b || forced <= 2) && forced <= 6) return forced;
    if (any_b) {
        if (ok(2)) return 2;
        if (!cv && ok(1)) return 1;
        return 0;
    }
    // FP64 blocks of 8 keep the register tile at 8 x 4 values.
    const int pref_real[3] = {4, 2, 1};
    const int pref_cplx[3] = {4, 6, 2};
    const int* pref = cv ? pref_cplx : pref_real;
    (void)dbl;
    if (block_size == 1) {
        // Scalar rows: the first width whose W / V threads per row tile a
        // warp exactly (measured on the twisted-bilayer transport panel,
        // complex W = 96: V = 6, 16 threads per row, 5 % faster than V = 4's
        // 24, which leaves rows straddling warps).
        for (int i = 0; i < 3; ++i) {
            const int L = ok(pref[i]) ? W / pref[i] : 0;
            if (L && (32 % L == 0 || L % 32 == 0)) return pref[i];
        }
    }
    for (int i = 0; i < 3; ++i)
        if (ok(pref[i])) return pref[i];
    return 0;
}

constexpr int kNotApplicable = 1000;

// RSATB_STEP_KERNEL=v1|staged|rowsplit|bulk|narrow|dmma|tf32|generic forces one kernel family
// (tuning and A/B tests); unset picks by shape and precision.
inline int env_kernel() {
    const char* s = std::getenv("RSATB_STEP_KERNEL");
    if (!s) return 0;
    if (s[0] == 'v' && s[1] == '1') return 1;
    if (s[0] == 's') return 2;
    if (s[0] == 'r') return 3;
    if (s[0] == 'b') return 4;
    if (s[0] == 'n') return 5;
    if (s[0] == 'd') return 6;
    if (s[0] == 't') return 7;
    if (s[0] == 'g') return 8;  // the register kernel
    return 0;
}
inline bool env_force_v1() { return env_kernel() == 1; }

template <typename VT, int B, int KL, int WW, bool CV>
int launch_rowsplit_k(rsatb_context* ctx, StepArgs& a) {
    constexpr int UNROLL = WW <= 8 ? 4 : 2;
    auto kernel = cheb_step_rowsplit<VT, B, KL, WW, CV, UNROLL>;
    const int threads = 256;
    const int ndots = a.dot_mode == DOT_NONE ? 0 : 2;
    const size_t smem = size_t(ndots) * threads * (WW / KL) * sizeof(double);
    const int64_t need = (a.n_block_rows + 7) / 8;
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, smem);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, smem, ctx->stream>>>(a);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

// Narrow real-matrix panels (W in {4, 8, 16}) with blocks of 5 or 8.
template <typename VT, bool CM, bool CV>
int launch_rowsplit(rsatb_context* ctx, int block_size, StepArgs& a) {
    if constexpr (CM) {
        return kNotApplicable;
    } else {
        if (a.W == 16) {
            if (block_size == 8) return launch_rowsplit_k<VT, 8, 4, 16, CV>(ctx, a);
            if (block_size == 5) return launch_rowsplit_k<VT, 5, 4, 16, CV>(ctx, a);
        } else if (a.W == 8) {
            if (block_size == 8) return launch_rowsplit_k<VT, 8, 4, 8, CV>(ctx, a);
            if (block_size == 5) return launch_rowsplit_k<VT, 5, 4, 8, CV>(ctx, a);
        } else if (a.W == 4 && !CV) {
            if (block_size == 8) return launch_rowsplit_k<VT, 8, 4, 4, false>(ctx, a);
            if (block_size == 5) return launch_rowsplit_k<VT, 5, 4, 4, false>(ctx, a);
        }
        return kNotApplicable;
    }
}

// The cp.async-staged kernel (cheb_staged.cuh); kNotApplicable when the
// panel width has no staged mapping (the caller falls back to the
// register kernel).
template <typename VT, typename MT, int B, int V, bool CM, bool CV>
int launch_staged(rsatb_context* ctx, StepArgs& a) {
    constexpr int STAGES = 3;
    const int L = a.W / V;
    int Lp, n_chunks;
    if (L <= 32) {
        if (32 % L) return kNotApplicable;
        Lp = L;
        n_chunks = 1;
    } else {
        if (L % 32) return kNotApplicable;
        Lp = 32;
        n_chunks = L / 32;
    }
    const int spw = 32 / Lp;
    const int wb = staged_warp_bytes<VT, MT, B, V, CM, STAGES>(spw);
    int warps = 8;
    while (warps > n_chunks && warps > 1 && warps * wb > 112 * 1024) warps /= 2;
    if (warps % n_chunks) return kNotApplicable;
    const int threads = warps * 32;
    const int ndots = a.dot_mode == DOT_NONE ? 0 : 2;
    size_t smem = size_t(warps) * wb;
    const size_t red = size_t(ndots) * threads * V * sizeof(double);
    if (red > smem) smem = red;
    if (smem > 227 * 1024) return kNotApplicable;
    auto kernel = cheb_step_staged<VT, MT, B, V, CM, CV, STAGES>;
    // Raise the dynamic shared-memory limit of this instantiation as far as
    // this launch needs (a process-wide setting of the function).  Opted in
    // from the first launch: the kernel also holds static shared memory (the
    // dot finish), so 48 KB of dynamic memory alone already exceeds the
    // default limit.
    static size_t attr_bytes = 0;
    if (smem > attr_bytes) {
        cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(smem));
        if (err != cudaSuccess) {
            cudaGetLastError();
            return kNotApplicable;  // the register kernel needs no opt-in
        }
        attr_bytes = smem;
    }
    const int64_t items = a.n_block_rows * n_chunks;
    const int64_t per_cta = int64_t(warps) * spw;
    const int64_t need = (items + per_cta - 1) / per_cta;
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, smem);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, smem, ctx->stream>>>(a, Lp, n_chunks);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

template <typename VT, typename MT, int B, bool CM, bool CV>
int launch_staged_v(rsatb_context* ctx, int V, StepArgs& a) {
    switch (V) {
        case 1:
            if constexpr (!CV) return launch_staged<VT, MT, B, 1, CM, CV>(ctx, a);
            break;
        case 2: return launch_staged<VT, MT, B, 2, CM, CV>(ctx, a);
        case 4: return launch_staged<VT, MT, B, 4, CM, CV>(ctx, a);
        case 6:
            if constexpr (CV) return launch_staged<VT, MT, B, 6, CM, CV>(ctx, a);
            break;
    }
    return kNotApplicable;
}

// V for the staged kernel: FP64 blocks of 8 take 2 values per thread (the
// register tile stays near 100 registers), everything else 4 when it fits.
inline int pick_v_staged(int W, bool cv, int block_size, bool dbl) {
    const int forced = env_v();
    auto ok = [&](int v) {
        if (v <= 0 || v > 6 || W % v) return false;
        if (cv && v % 2) return false;
        const int L = W / v;
        return (L <= 32 && 32 % L == 0) || (L > 32 && L % 32 == 0 && L <= 256);
    };
    if (forced && ok(forced)) return forced;
    const int real64[3] = {2, 4, 1}, real32[3] = {4, 2, 1}, cplx[3] = {4, 2, 6},
              cplx64[3] = {2, 4, 6};
    const int* pref = cv ? ((dbl && block_size == 8) ? cplx64 : cplx)
                         : ((dbl && block_size == 8) ? real64 : real32);
    for (int i = 0; i < 3; ++i)
        if (ok(pref[i])) return pref[i];
    return 0;
}

// Ring depth of the bulk-copy kernel (RSATB_BULK_NS=3 overrides the 2
// stages), where its X rows come from (RSATB_BULK_X=smem: through the ring
// too; default: L1-cached global loads) and its register budget
// (RSATB_BULK_OCC=4: sized for 4 resident CTAs per SM instead of 3).
inline int bulk_stages() {
    const char* s = std::getenv("RSATB_BULK_NS");
    const int n = s ? std::atoi(s) : 2;
    return (n == 3 || n == 4) ? n : 2;
}
inline bool bulk_x_global() {
    const char* s = std::getenv("RSATB_BULK_X");
    return !(s && s[0] == 's');
}
inline bool bulk_occ4() {
    const char* s = std::getenv("RSATB_BULK_OCC");
    return s && std::atoi(s) == 4;
}
// A from the duplicated transposed slot (DUP): the default at W = 256,
// where it measured 0.92 against 1.11 ms per launch on the diamond 16^3
// BSR; at W = 32 to 128 the row-major slot is faster (0.427 against
// 0.451 ms at W = 128).  RSATB_BULK_A=dup|row forces one (A/B only).
inline bool bulk_a_dup(int W) {
    const char* s = std::getenv("RSATB_BULK_A");
    if (s && s[0] == 'd') return true;
    if (s && s[0] == 'r') return false;
    return W >= 256;
}

template <int W, bool CV, int NS, bool XG, int MINB, bool DUP = false>
int launch_bulk_k(rsatb_context* ctx, StepArgs& a) {
    using Sh = BulkShape<W, XG>;
    auto kernel = cheb_step_bulk<W, CV, NS, XG, MINB, DUP>;
    const int threads = kBulkWarps * 32;
    const size_t smem = bulk_smem_bytes<W, XG, NS>();
    if (smem > 227 * 1024) return kNotApplicable;
    // Raise the dynamic shared-memory limit of this instantiation once.
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)) != cudaSuccess) {
            cudaGetLastError();
            return kNotApplicable;
        }
        attr_set = true;
    }
    const int64_t groups = (a.n_block_rows + Sh::S - 1) / Sh::S;
    const int64_t need = (groups + kBulkWarps - 1) / kBulkWarps;
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, smem);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (grid > int64_t(ctx->sm_count) * 8) grid = int64_t(ctx->sm_count) * 8;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, smem, ctx->stream>>>(a);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

template <int W, bool CV>
int launch_bulk_w(rsatb_context* ctx, StepArgs& a) {
    // RSATB_TEST_BULK_WAIT=1: run only the wait that cannot complete (tests
    // of the bounded-wait fault report).
    const char* wc = std::getenv("RSATB_TEST_BULK_WAIT");
    a.wait_check = (wc && wc[0] == '1') ? 1 : 0;
    const int ns = bulk_stages();
    if (!bulk_x_global())
        return ns == 3 ? launch_bulk_k<W, CV, 3, false, 2>(ctx, a)
                       : launch_bulk_k<W, CV, 2, false, 3>(ctx, a);
    if (bulk_occ4()) return launch_bulk_k<W, CV, 2, true, 4>(ctx, a);
    const bool dup = bulk_a_dup(W);
    if (ns == 3)
        return dup ? launch_bulk_k<W, CV, 3, true, 3, true>(ctx, a)
                   : launch_bulk_k<W, CV, 3, true, 3, false>(ctx, a);
    if (ns == 4)
        return dup ? launch_bulk_k<W, CV, 4, true, 3, true>(ctx, a)
                   : launch_bulk_k<W, CV, 4, true, 3, false>(ctx, a);
    return dup ? launch_bulk_k<W, CV, 2, true, 3, true>(ctx, a)
               : launch_bulk_k<W, CV, 2, true, 3, false>(ctx, a);
}

// Ring depth of the narrow-panel kernel (RSATB_NARROW_NS: 2 or 3).
inline int narrow_stages() {
    const char* s = std::getenv("RSATB_NARROW_NS");
    return (s && std::atoi(s) == 3) ? 3 : 2;
}

template <typename VT, int W, bool CV, int NS>
int launch_narrow_k(rsatb_context* ctx, StepArgs& a) {
    using Sh = NarrowShape<VT, W>;
    auto kernel = cheb_step_narrow<VT, W, CV, NS>;
    const int threads = kNarrowWarps * 32;
    // The ring, or the dots reduction that reuses it, whichever is larger.
    constexpr size_t ring = narrow_smem_bytes<VT, W, NS>();
    constexpr size_t red_max = 2 * size_t(kNarrowWarps) * 32 * Sh::V * sizeof(double);
    constexpr size_t smem = ring > red_max ? ring : red_max;
    if (smem > 200 * 1024) return kNotApplicable;
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)) != cudaSuccess) {
            cudaGetLastError();
            return kNotApplicable;
        }
        attr_set = true;
    }
    const int64_t groups = (a.n_block_rows + Sh::S - 1) / Sh::S;
    const int64_t need = (groups + kNarrowWarps - 1) / kNarrowWarps;
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, smem);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (grid > int64_t(ctx->sm_count) * 8) grid = int64_t(ctx->sm_count) * 8;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, smem, ctx->stream>>>(a);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

template <typename VT, int W, bool CV>
int launch_narrow_w(rsatb_context* ctx, StepArgs& a) {
    return narrow_stages() == 3 ? launch_narrow_k<VT, W, CV, 3>(ctx, a)
                                : launch_narrow_k<VT, W, CV, 2>(ctx, a);
}

// Blocks of a row loaded together by the tensor-core kernel at W <= 32
// (RSATB_DMMA_U: 2, 4 or 8; unset: by width).
inline int dmma_u() {
    const char* s = std::getenv("RSATB_DMMA_U");
    const int u = s ? std::atoi(s) : 0;
    return (u == 2 || u == 4 || u == 8) ? u : 0;
}

template <typename VT, int W, bool CV, int UU>
int launch_dmma_u(rsatb_context* ctx, StepArgs& a) {
    auto kernel = cheb_step_dmma<VT, W, CV, UU>;
    constexpr int kWarps = dmma_warps<VT>();
    const int threads = kWarps * 32;
    const int64_t need = (a.n_block_rows + kWarps - 1) / kWarps;
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, 0);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (grid > int64_t(ctx->sm_count) * 8) grid = int64_t(ctx->sm_count) * 8;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, 0, ctx->stream>>>(a);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

template <typename VT, int W, bool CV>
int launch_dmma_k(rsatb_context* ctx, StepArgs& a) {
    if constexpr (W <= 32) {
        switch (dmma_u()) {
            case 2: return launch_dmma_u<VT, W, CV, 2>(ctx, a);
            case 4: return launch_dmma_u<VT, W, CV, 4>(ctx, a);
            case 8: return launch_dmma_u<VT, W, CV, 8>(ctx, a);
        }
    }
    return launch_dmma_u<VT, W, CV, 0>(ctx, a);
}

// Panels on the FP64 tensor cores: real 8x8 blocks, W a multiple of 8 up
// to 256 (complex panels: W = 2R); FP32 panels at W <= 32 only (wider ones
// are compute-bound, where the FP32 FMA kernels are faster); kNotApplicable
// otherwise.
template <typename VT, bool CV>
int launch_dmma(rsatb_context* ctx, StepArgs& a) {
    if (sizeof(VT) == 4 && a.W > 32) return kNotApplicable;
    switch (a.W) {
        case 8: return launch_dmma_k<VT, 8, CV>(ctx, a);
        case 16: return launch_dmma_k<VT, 16, CV>(ctx, a);
        case 32: return launch_dmma_k<VT, 32, CV>(ctx, a);
        case 64:
            if constexpr (sizeof(VT) == 8) return launch_dmma_k<VT, 64, CV>(ctx, a);
            break;
        case 128:
            if constexpr (sizeof(VT) == 8) return launch_dmma_k<VT, 128, CV>(ctx, a);
            break;
        case 256:
            if constexpr (sizeof(VT) == 8) return launch_dmma_k<VT, 256, CV>(ctx, a);
            break;
    }
    return kNotApplicable;
}

// Real 8x8 blocks, W in {4, 8, 16}, 16-byte aligned values and operand;
// kNotApplicable otherwise.
template <typename VT, bool CV>
int launch_narrow(rsatb_context* ctx, StepArgs& a) {
    if ((reinterpret_cast<uintptr_t>(a.vals) | reinterpret_cast<uintptr_t>(a.in)) & 15u)
        return kNotApplicable;
    switch (a.W) {
        case 4:
            if constexpr (!CV) return launch_narrow_w<VT, 4, CV>(ctx, a);
            break;
        case 8: return launch_narrow_w<VT, 8, CV>(ctx, a);
        case 16: return launch_narrow_w<VT, 16, CV>(ctx, a);
    }
    return kNotApplicable;
}

// FP32 panels, real 8x8 blocks, W in {8, 16, 32, 64, 128, 256}, 16-byte
// aligned values and operand; kNotApplicable otherwise.
template <bool CV>
int launch_bulk(rsatb_context* ctx, StepArgs& a) {
    if ((reinterpret_cast<uintptr_t>(a.vals) | reinterpret_cast<uintptr_t>(a.in)) & 15u)
        return kNotApplicable;
    switch (a.W) {
        case 8:
            if constexpr (!CV) return launch_bulk_w<8, CV>(ctx, a);
            break;
        case 16: return launch_bulk_w<16, CV>(ctx, a);
        case 32: return launch_bulk_w<32, CV>(ctx, a);
        case 64: return launch_bulk_w<64, CV>(ctx, a);
        case 128: return launch_bulk_w<128, CV>(ctx, a);
        case 256: return launch_bulk_w<256, CV>(ctx, a);
    }
    return kNotApplicable;
}

template <int W, bool CV, int P, int MINB>
int launch_tf32_k(rsatb_context* ctx, StepArgs& a) {
    auto kernel = cheb_step_tf32<W, CV, P, MINB>;
    const int threads = kTf32Warps * 32;
    const int64_t need = (a.n_block_rows + kTf32Warps / 2 - 1) / (kTf32Warps / 2);
    const int per_sm = occupancy(reinterpret_cast<const void*>(kernel), threads, 0);
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kernel<<<unsigned(grid), threads, 0, ctx->stream>>>(a);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

// Split-TF32 tensor-core kernel: FP32 panels, real 8x8 blocks, W in {64,
// 128, 256}, 16-byte aligned values and operand; kNotApplicable otherwise.
template <bool CV>
int launch_tf32(rsatb_context* ctx, StepArgs& a) {
    if ((reinterpret_cast<uintptr_t>(a.vals) | reinterpret_cast<uintptr_t>(a.in)) & 15u)
        return kNotApplicable;
    // RSATB_TF32_SHAPE=p3: three blocks in flight at one CTA per SM less.
    const char* s = std::getenv("RSATB_TF32_SHAPE");
    const bool p3 = s && s[0] == 'p' && s[1] == '3';
    switch (a.W) {
        case 64:
            return p3 ? launch_tf32_k<64, CV, 3, 2>(ctx, a) : launch_tf32_k<64, CV, 2, 3>(ctx, a);
        case 128:
            return p3 ? launch_tf32_k<128, CV, 3, 1>(ctx, a) : launch_tf32_k<128, CV, 2, 2>(ctx, a);
        case 256:
            return p3 ? launch_tf32_k<256, CV, 3, 1>(ctx, a) : launch_tf32_k<256, CV, 2, 1>(ctx, a);
    }
    return kNotApplicable;
}

template <typename VT, typename MT, int B, bool CM, bool CV>
int launch_b(rsatb_context* ctx, int V, int64_t rows, StepArgs& a);

template <typename VT, typename MT, int B, bool CM, bool CV>
int launch_b(rsatb_context* ctx, int V, int64_t rows, StepArgs& a) {
    switch (V) {
        case 1:
            if constexpr (!CV) return launch(ctx, cheb_step_kernel<VT, MT, B, 1, CM, CV>, 1, rows, a);
            break;
        case 2: return launch(ctx, cheb_step_kernel<VT, MT, B, 2, CM, CV>, 2, rows, a);
        case 4: return launch(ctx, cheb_step_kernel<VT, MT, B, 4, CM, CV>, 4, rows, a);
        case 6:
            if constexpr (CV) return launch(ctx, cheb_step_kernel<VT, MT, B, 6, CM, CV>, 6, rows, a);
            break;
    }
    return set_error(RSATB_NOT_SUPPORTED, "no step kernel for V=%d", V);
}

template <typename VT, typename MT, bool CM, bool CV>
int launch_typed(rsatb_context* ctx, int block_size, StepArgs& a) {
    const bool special = block_size == 1 || block_size == 5 || block_size == 8;
    const int V = pick_v(a.W, CV, !special, block_size, sizeof(VT) == 8);
    if (V == 0)
        return set_error(RSATB_NOT_SUPPORTED,
                         "panel width %d (real values per row) has no thread mapping; widths up "
                         "to 1536 are supported", a.W);
    const int64_t rows = a.n_block_rows;
    const int forced = env_kernel();
    if (forced == 3 && (block_size == 5 || block_size == 8)) {
        const int st = launch_rowsplit<VT, CM, CV>(ctx, block_size, a);
        if (st != kNotApplicable) return st;
    }
    if constexpr (!CM) {
        // FP64 tensor-core kernel, blocks of 8: the default for FP64 panels
        // and for FP32 panels of W <= 16 (measured on the diamond 8x8 BSR,
        // B200: FP64 R = 8 / 16 / 32 / 128 take 0.093 / 0.158 / 0.267 /
        // 1.01 ms against 0.226 / 0.213 / 0.349 / 1.22 for the staged
        // kernel; FP32 R = 8 / 16 take 0.078 / 0.109 ms against 0.103 /
        // 0.119 for the register kernel).
        const bool want = forced == 6 || (forced == 0 && (sizeof(VT) == 8 || a.W <= 16));
        if (block_size == 8 && want) {
            const int st = launch_dmma<VT, CV>(ctx, a);
            if (st != kNotApplicable) return st;
        }
    }
    if constexpr (!CM) {
        // Narrow-panel lock-step kernel: blocks of 8, W <= 16 (when forced).
        if (block_size == 8 && forced == 5) {
            const int st = launch_narrow<VT, CV>(ctx, a);
            if (st != kNotApplicable) return st;
        }
    }
    if constexpr (sizeof(VT) == 4 && !CM) {
        // Split-TF32 tensor-core kernel (when forced).
        if (block_size == 8 && forced == 7) {
            const int st = launch_tf32<CV>(ctx, a);
            if (st != kNotApplicable) return st;
        }
    }
    if constexpr (sizeof(VT) == 4 && !CM) {
        // Bulk-copy kernel: FP32, blocks of 8, panels of 32 to 256 values
        // by default (every width when forced).
        const bool wide = a.W >= 32;
        if (block_size == 8 && (forced == 4 || (forced == 0 && wide))) {
            const int st = launch_bulk<CV>(ctx, a);
            if (st != kNotApplicable) return st;
        }
    }
    // Measured choice (diamond 8x8 blocks, B200), after the tensor-core and
    // bulk-copy kernels above: FP64 takes the staged kernel (other block
    // sizes), FP32 the staged kernel for complex panels of W = 16 and the
    // register kernel otherwise.  Scalar rows take the register kernel in
    // both precisions (twisted-bilayer transport recurrence: FP64 complex
    // W = 32 and 96, 225 against 519 ms for 256 moments; FP32 complex W = 16
    // and 48, 175 against 259 ms for 512).
    const bool want_staged =
        forced == 2 ||
        (forced == 0 && block_size != 1 && (sizeof(VT) == 8 || (a.W == 16 && CV)));
    if (special && want_staged) {
        const int Vs = pick_v_staged(a.W, CV, block_size, sizeof(VT) == 8);
        int st = kNotApplicable;
        if (Vs) {
            switch (block_size) {
                case 1: st = launch_staged_v<VT, MT, 1, CM, CV>(ctx, Vs, a); break;
                case 5: st = launch_staged_v<VT, MT, 5, CM, CV>(ctx, Vs, a); break;
                case 8: st = launch_staged_v<VT, MT, 8, CM, CV>(ctx, Vs, a); break;
            }
        }
        if (st != kNotApplicable) return st;
    }
    switch (block_size) {
        case 1: return launch_b<VT, MT, 1, CM, CV>(ctx, V, rows, a);
        case 5: return launch_b<VT, MT, 5, CM, CV>(ctx, V, rows, a);
        case 8: return launch_b<VT, MT, 8, CM, CV>(ctx, V, rows, a);
        default:
            if (V == 2) return launch(ctx, cheb_step_kernel_any_b<VT, MT, 2, CM, CV>, 2, rows, a);
            if constexpr (!CV)
                return launch(ctx, cheb_step_kernel_any_b<VT, MT, 1, CM, CV>, 1, rows, a);
            return set_error(RSATB_NOT_SUPPORTED, "no generic step kernel for V=%d", V);
    }
}

template <typename VT>
int launch_step_precision(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vec_dtype,
                          StepArgs& a) {
    const bool cm = dtype_is_complex(A->dtype);
    const bool cv = dtype_is_complex(vec_dtype);
    if (cm && !cv)
        return set_error(RSATB_INVALID_ARGUMENT, "a complex matrix needs a complex multivector");
    if ((A->flags & RSATB_BSR_IMAGINARY_UNIT) && !cv)
        return set_error(RSATB_INVALID_ARGUMENT,
                         "an imaginary-unit matrix needs a complex multivector");
    a.imag = (A->flags & RSATB_BSR_IMAGINARY_UNIT) ? 1 : 0;
    a.n_block_rows = A->n_block_rows;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.vals = A->values;
    a.block_size = A->block_size;
    if (cm) return launch_typed<VT, VT, true, true>(ctx, A->block_size, a);
    if (cv) return launch_typed<VT, VT, false, true>(ctx, A->block_size, a);
    return launch_typed<VT, VT, false, false>(ctx, A->block_size, a);
}

template <typename VT>
int launch_coldot_precision(rsatb_context* ctx, int vec_dtype, int64_t n_rows, StepArgs& a) {
    const bool cv = dtype_is_complex(vec_dtype);
    const int V = pick_v(a.W, cv, false, 1, sizeof(VT) == 8);
    if (V == 0) return set_error(RSATB_NOT_SUPPORTED, "panel width %d not supported", a.W);
    a.dot_mode = DOT_PLAIN;
    a.n_block_rows = n_rows;
    if (cv) {
        switch (V) {
            case 2: return launch(ctx, coldot_kernel<VT, 2, true>, 2, n_rows, a);
            case 4: return launch(ctx, coldot_kernel<VT, 4, true>, 4, n_rows, a);
            case 6: return launch(ctx, coldot_kernel<VT, 6, true>, 6, n_rows, a);
        }
    } else {
        switch (V) {
            case 1: return launch(ctx, coldot_kernel<VT, 1, false>, 1, n_rows, a);
            case 2: return launch(ctx, coldot_kernel<VT, 2, false>, 2, n_rows, a);
            case 4: return launch(ctx, coldot_kernel<VT, 4, false>, 4, n_rows, a);
        }
    }
    return set_error(RSATB_NOT_SUPPORTED, "no dot kernel for V=%d", V);
}

}  // namespace step_detail
}  // namespace rsatb_b200
