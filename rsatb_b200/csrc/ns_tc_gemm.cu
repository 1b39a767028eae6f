// Batched C = A B^T on the sm_100a tensor cores (tcgen05, kind::tf32) for
// the Newton-Schulz inverse square root: one 128 x nt tile of one problem
// per work item, persistent CTAs striding over the items.
//
// CTA = 4 warps.  Thread 0 is the TMA producer: per K chunk of 32 values it
// loads the A tile (128 rows) and the B tile (nt rows) of the chunk, as the
// TF32 "hi" arrays and, for split precision, the "lo" residual arrays, into
// a 2-stage ring of 128-byte-swizzled shared-memory tiles.  Thread 32
// issues the MMAs: per chunk four K=8 steps, each hi*hi (+ hi*lo + lo*hi
// when split), accumulating in FP32 in TMEM (128 lanes x nt columns), and
// commits each stage back to the producer.  After the last chunk all four
// warps read the accumulator out of TMEM (warp w owns rows 32w..32w+31) and
// run the epilogue: the Newton-Schulz polynomial or the residual
// ||C - I||_F^2, the TF32 hi/lo split of the result and, optionally, its
// FP64 value.
#include "ns_batched.cuh"
#include "umma.cuh"

#include <cudaTypedefs.h>
#include <cstdlib>
#include <mutex>

namespace rsatb_b200 {
namespace ns {
namespace {

constexpr int kStages = 2;
constexpr int kTileA = 128 * 128;  // bytes of one A tile: 128 rows x 32 fp32
constexpr int kTileB = 256 * 128;  // bytes of one B tile: up to 256 rows
constexpr int kStageBytes = 2 * kTileA + 2 * kTileB;
constexpr int kSmemBytes = kStages * kStageBytes + 1024;  // + alignment slack
constexpr uint32_t kTmemCols = 256;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ void record_error(unsigned* error, unsigned code) {
    if (error) atomicOr(error, code);
}

// Stores one thread's 16 consecutive values of C (row `row`, columns col0..
// col0 + 15 of the padded problem): the hi/lo pair and the optional FP64
// copy at (row, col), and the optional transposed hi/lo at (col, row); with
// args.sym only the upper triangle (col >= row) is stored, each element
// also at (col, row), so C leaves exactly symmetric.  The transposed and
// mirrored stores of a warp (32 consecutive rows, one column) are
// coalesced.
// X (hi + lo) at 16 consecutive elements for the polynomial epilogue, as
// 128-bit loads.
__device__ __forceinline__ void load_x16(const TcArgs& args, int64_t base, float (&xe)[16]) {
    const float4* h = reinterpret_cast<const float4*>(args.xe_hi + base);
    const float4* l = reinterpret_cast<const float4*>(args.xe_lo + base);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 a = h[q], b = l[q];
        xe[4 * q] = a.x + b.x;
        xe[4 * q + 1] = a.y + b.y;
        xe[4 * q + 2] = a.z + b.z;
        xe[4 * q + 3] = a.w + b.w;
    }
}

__device__ __forceinline__ void store_rows(const TcArgs& args, int64_t base,
                                           const float (&hi)[16], const float (&lo)[16]) {
    if (args.c_hi) {
        float4* ch = reinterpret_cast<float4*>(args.c_hi + base);
        float4* cl = reinterpret_cast<float4*>(args.c_lo + base);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ch[q] = make_float4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
            cl[q] = make_float4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
        }
    }
    if (args.c64) {
        double2* cd = reinterpret_cast<double2*>(args.c64 + base);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            cd[q] = make_double2(double(hi[2 * q]) + double(lo[2 * q]),
                                 double(hi[2 * q + 1]) + double(lo[2 * q + 1]));
    }
}

__device__ __forceinline__ void store_chunk(const TcArgs& args, const Prob& pr, int row, int col0,
                                            const float (&hi)[16], const float (&lo)[16]) {
    const int np = pr.n_pad;
    const int64_t base = pr.off + int64_t(row) * np + col0;
    if (args.sym) {
        if (col0 + 15 < row) return;  // below the diagonal: the mirror of another thread's
        if (col0 >= row) {
            store_rows(args, base, hi, lo);  // the whole chunk is on or above the diagonal
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                if (col0 + j < row) continue;
                args.c_hi[base + j] = hi[j];
                args.c_lo[base + j] = lo[j];
                if (args.c64) args.c64[base + j] = double(hi[j]) + double(lo[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {  // mirror: for fixed j a warp writes 32 consecutive rows
            const int col = col0 + j;
            if (col <= row) continue;
            const int64_t t = pr.off + int64_t(col) * np + row;
            args.c_hi[t] = hi[j];
            args.c_lo[t] = lo[j];
            if (args.c64) args.c64[t] = double(hi[j]) + double(lo[j]);
        }
        return;
    }
    store_rows(args, base, hi, lo);
    if (args.ct_hi) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int64_t t = pr.off + int64_t(col0 + j) * np + row;
            args.ct_hi[t] = hi[j];
            args.ct_lo[t] = lo[j];
        }
    }
}

__global__ void __launch_bounds__(128, 1)
    tc_gemm_kernel(const __grid_constant__ TcMaps maps, const TcArgs args) {
    using namespace umma;
    if (args.live && *args.live == 0) return;  // every problem has stopped
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kStages];
    __shared__ __align__(8) uint64_t empty[kStages];
    __shared__ __align__(8) uint64_t done;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        tmem_alloc(&tmem_base, kTmemCols);
        tmem_relinquish();
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        fence_mbarrier_init();
        abort_flag = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    uint32_t chunk_base = 0;  // K chunks this CTA has streamed (ring position)
    uint32_t n_done = 0;      // tiles this CTA has finished (phase of `done`)
    for (int it = blockIdx.x; it < args.n_items; it += gridDim.x) {
        const TcItem item = args.items[it];
        if (!args.state[item.p].active) continue;
        const Prob pr = args.probs[item.p];
        const int nk = pr.n_pad / 32;
        const uint32_t tx_bytes = uint32_t(kTileA + item.nt * 128) * (args.split ? 2u : 1u);

        if (threadIdx.x == 0) {
            // ---- TMA producer
            const CUtensorMap* ah = &maps.a_hi[item.bucket];
            const CUtensorMap* al = &maps.a_lo[item.bucket];
            const CUtensorMap* bh = &maps.b_hi[item.bucket];
            const CUtensorMap* bl = &maps.b_lo[item.bucket];
            for (int kc = 0; kc < nk; ++kc) {
                const uint32_t g = chunk_base + kc;
                const int s = int(g % kStages);
                const uint32_t ph = (g / kStages) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u, kWaitLimitNs)) {
                    record_error(args.error, 1u);
                    abort_flag = 1;
                    break;
                }
                uint8_t* st = smem + s * kStageBytes;
                mbar_arrive_expect_tx(&full[s], tx_bytes);
                tma_load_3d(st, ah, &full[s], kc * 32, item.m0, item.z);
                tma_load_3d(st + 2 * kTileA, bh, &full[s], kc * 32, item.n0, item.z);
                if (args.split) {
                    tma_load_3d(st + kTileA, al, &full[s], kc * 32, item.m0, item.z);
                    tma_load_3d(st + 2 * kTileA + kTileB, bl, &full[s], kc * 32, item.n0,
                                item.z);
                }
            }
        } else if (threadIdx.x == 32) {
            // ---- MMA issuer
            const uint32_t idesc = idesc_tf32(128, item.nt);
            bool ok = true;
            for (int kc = 0; kc < nk; ++kc) {
                const uint32_t g = chunk_base + kc;
                const int s = int(g % kStages);
                const uint32_t ph = (g / kStages) & 1u;
                if (!mbar_wait(&full[s], ph, kWaitLimitNs)) {
                    record_error(args.error, 2u);
                    abort_flag = 1;
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a_hi = smem_u32(smem + s * kStageBytes);
                const uint32_t a_lo = a_hi + kTileA;
                const uint32_t b_hi = a_hi + 2 * kTileA;
                const uint32_t b_lo = b_hi + kTileB;
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const uint32_t ko = kk * 32;  // 8 TF32 values = 32 bytes along K
                    const uint64_t dah = desc_kmajor_sw128(a_hi + ko);
                    const uint64_t dbh = desc_kmajor_sw128(b_hi + ko);
                    mma_tf32(tmem, dah, dbh, idesc, (kc | kk) ? 1u : 0u);
                    if (args.split) {
                        mma_tf32(tmem, dah, desc_kmajor_sw128(b_lo + ko), idesc, 1u);
                        mma_tf32(tmem, desc_kmajor_sw128(a_lo + ko), dbh, idesc, 1u);
                    }
                }
                mma_commit(&empty[s]);
            }
            if (ok) mma_commit(&done);
        }
        chunk_base += nk;

        // ---- epilogue, all 128 threads
        __syncwarp();
        const bool ok = mbar_wait(&done, n_done & 1u, kWaitLimitNs);
        ++n_done;
        if (!ok) {
            if (lane == 0) record_error(args.error, 4u);
            abort_flag = 1;
        }
        tc_fence_after();
        if (ok) {
            const int row = item.m0 + warp * 32 + lane;
            const bool in_mat = row < pr.n_pad;
            const bool vrow = row < pr.n;
            const int np = pr.n_pad;
            const PolyCoef pc = poly_coef(args.mode == EPI_POLY && args.state[item.p].lift);
            double r2 = 0.0;
            for (int c = 0; c < item.nt; c += 16) {
                float v[16];
                tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c), v);
                const int col0 = item.n0 + c;
                if (!in_mat || col0 >= np) continue;
                const int64_t base = pr.off + int64_t(row) * np + col0;
                float hi[16], lo[16], xe[16];
                if (args.mode == EPI_POLY) load_x16(args, base, xe);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = col0 + j;
                    const bool valid = vrow && col < pr.n;
                    float x = v[j];
                    if (args.mode == EPI_POLY)
                        x = fmaf(pc.c, x, fmaf(pc.b, xe[j], row == col ? pc.a : 0.0f));
                    if (!valid) x = 0.0f;
                    if (args.mode == EPI_RESID && valid && (!args.sym || col >= row)) {
                        const double d = double(x) - (row == col ? 1.0 : 0.0);
                        r2 += (args.sym && col > row) ? 2.0 * d * d : d * d;
                    }
                    hi[j] = to_tf32(x);
                    lo[j] = x - hi[j];
                }
                store_chunk(args, pr, row, col0, hi, lo);
            }
            if (args.mode == EPI_RESID) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
                if (lane == 0 && r2 != 0.0) atomicAdd(args.res2 + item.p, r2);
            }
        }
        tc_fence_before();
        __syncthreads();
        if (abort_flag) break;
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// ---------------------------------------------------------------------------
// Warp-specialised variant: warp 0 is the TMA producer, warp 1 the MMA
// issuer (and TMEM owner), warps 2-9 the epilogue (two per TMEM lane
// quarter).  A 3-stage ring of
// 64 KB stages (A hi/lo and B hi/lo, K chunk 32, N tile <= 128) feeds the
// MMAs; the accumulator is double-buffered in TMEM (2 x 128 columns), so
// the epilogue of one tile overlaps the main loop of the next.
constexpr int kWsStages = 3;
constexpr int kWsTileB = 128 * 128;                 // B tile: up to 128 rows
constexpr int kWsStageBytes = 2 * kTileA + 2 * kWsTileB;
constexpr int kWsSmemBytes = kWsStages * kWsStageBytes + 1024;
constexpr uint32_t kWsTmemCols = 256;               // two 128-column accumulators

__device__ __forceinline__ void ws_epilogue(const TcArgs& args, const TcItem& item,
                                            const Prob& pr, uint32_t tacc, int quarter,
                                            int half, int lane) {
    using namespace umma;
    const int row = item.m0 + quarter * 32 + lane;
    const bool in_mat = row < pr.n_pad;
    const bool vrow = row < pr.n;
    const int np = pr.n_pad;
    const PolyCoef pc = poly_coef(args.mode == EPI_POLY && args.state[item.p].lift);
    double r2 = 0.0;
    // Two warps share a TMEM lane quarter: they take alternate 16-column
    // chunks, the next chunk's TMEM load in flight while one is stored.
    const uint32_t lanes = tacc + (uint32_t(quarter * 32) << 16);
    uint32_t cur[16], nxt[16];
    if (16 * half < item.nt) {
        tmem_ld16_issue(lanes + uint32_t(16 * half), cur);
        tmem_wait_ld();
    }
    for (int c = 16 * half; c < item.nt; c += 32) {
        const bool more = c + 32 < item.nt;  // warp-uniform
        if (more) tmem_ld16_issue(lanes + uint32_t(c + 32), nxt);
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(cur[j]);
        const int col0 = item.n0 + c;
        if (in_mat && col0 < np) {
            const int64_t base = pr.off + int64_t(row) * np + col0;
            float hi[16], lo[16], xe[16];
            if (args.mode == EPI_POLY) load_x16(args, base, xe);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = col0 + j;
                const bool valid = vrow && col < pr.n;
                float x = v[j];
                if (args.mode == EPI_POLY)
                    x = fmaf(pc.c, x, fmaf(pc.b, xe[j], row == col ? pc.a : 0.0f));
                if (!valid) x = 0.0f;
                if (args.mode == EPI_RESID && valid && (!args.sym || col >= row)) {
                    const double d = double(x) - (row == col ? 1.0 : 0.0);
                    r2 += (args.sym && col > row) ? 2.0 * d * d : d * d;
                }
                hi[j] = to_tf32(x);
                lo[j] = x - hi[j];
            }
            store_chunk(args, pr, row, col0, hi, lo);
        }
        if (more) {  // the next chunk's load was in flight during the stores
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j) cur[j] = nxt[j];
        }
    }
    if (args.mode == EPI_RESID) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        if (lane == 0 && r2 != 0.0) atomicAdd(args.res2 + item.p, r2);
    }
}

// A work item with what every role needs of it, read one item ahead so the
// global loads of the next item overlap the current tile (all roles walk
// the same item sequence and skip the same inactive problems).
struct ItemView {
    TcItem item;
    Prob pr;
    int active;
};
__device__ __forceinline__ ItemView view_item(const TcArgs& args, int it) {
    ItemView v{};
    if (it < args.n_items) {
        v.item = args.items[it];
        v.active = args.state[v.item.p].active;
        v.pr = args.probs[v.item.p];
    }
    return v;
}

__global__ void __launch_bounds__(320, 1)
    tc_gemm_ws_kernel(const __grid_constant__ TcMaps maps, const TcArgs args) {
    using namespace umma;
    if (args.live && *args.live == 0) return;  // every problem has stopped
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kWsStages];
    __shared__ __align__(8) uint64_t empty[kWsStages];
    __shared__ __align__(8) uint64_t acc_full[2];
    __shared__ __align__(8) uint64_t acc_empty[2];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 1) {
        tmem_alloc(&tmem_base, kWsTmemCols);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kWsStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 8);  // one arrival per epilogue warp
        }
        fence_mbarrier_init();
        abort_flag = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer
            uint32_t g = 0;
            ItemView nx = view_item(args, blockIdx.x);
            for (int it = blockIdx.x; it < args.n_items && !abort_flag; it += gridDim.x) {
                const ItemView cur = nx;
                nx = view_item(args, it + gridDim.x);
                const TcItem item = cur.item;
                if (!cur.active) continue;
                const int nk = cur.pr.n_pad / 32;
                const uint32_t tx = uint32_t(kTileA + item.nt * 128) * (args.split ? 2u : 1u);
                for (int kc = 0; kc < nk; ++kc, ++g) {
                    const int s = int(g % kWsStages);
                    const uint32_t ph = (g / kWsStages) & 1u;
                    if (!mbar_wait(&empty[s], ph ^ 1u, kWaitLimitNs)) {
                        record_error(args.error, 1u);
                        abort_flag = 1;
                        break;
                    }
                    uint8_t* st = smem + s * kWsStageBytes;
                    mbar_arrive_expect_tx(&full[s], tx);
                    tma_load_3d(st, &maps.a_hi[item.bucket], &full[s], kc * 32, item.m0, item.z);
                    tma_load_3d(st + 2 * kTileA, &maps.b_hi[item.bucket], &full[s], kc * 32,
                                item.n0, item.z);
                    if (args.split) {
                        tma_load_3d(st + kTileA, &maps.a_lo[item.bucket], &full[s], kc * 32,
                                    item.m0, item.z);
                        tma_load_3d(st + 2 * kTileA + kWsTileB, &maps.b_lo[item.bucket], &full[s],
                                    kc * 32, item.n0, item.z);
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer
            uint32_t g = 0, t = 0;
            ItemView nx = view_item(args, blockIdx.x);
            for (int it = blockIdx.x; it < args.n_items && !abort_flag; it += gridDim.x) {
                const ItemView cur = nx;
                nx = view_item(args, it + gridDim.x);
                const TcItem item = cur.item;
                if (!cur.active) continue;
                const int nk = cur.pr.n_pad / 32;
                const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
                ++t;
                if (!mbar_wait(&acc_empty[b], tph ^ 1u, kWaitLimitNs)) {
                    record_error(args.error, 8u);
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t dacc = tmem + b * 128u;
                const uint32_t idesc = idesc_tf32(128, item.nt);
                bool ok = true;
                for (int kc = 0; kc < nk; ++kc, ++g) {
                    const int s = int(g % kWsStages);
                    const uint32_t ph = (g / kWsStages) & 1u;
                    if (!mbar_wait(&full[s], ph, kWaitLimitNs)) {
                        record_error(args.error, 2u);
                        abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_hi = smem_u32(smem + s * kWsStageBytes);
                    const uint32_t a_lo = a_hi + kTileA;
                    const uint32_t b_hi = a_hi + 2 * kTileA;
                    const uint32_t b_lo = b_hi + kWsTileB;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint32_t ko = kk * 32;
                        const uint64_t dah = desc_kmajor_sw128(a_hi + ko);
                        const uint64_t dbh = desc_kmajor_sw128(b_hi + ko);
                        mma_tf32(dacc, dah, dbh, idesc, (kc | kk) ? 1u : 0u);
                        if (args.split) {
                            mma_tf32(dacc, dah, desc_kmajor_sw128(b_lo + ko), idesc, 1u);
                            mma_tf32(dacc, desc_kmajor_sw128(a_lo + ko), dbh, idesc, 1u);
                        }
                    }
                    mma_commit(&empty[s]);
                }
                if (!ok) break;
                mma_commit(&acc_full[b]);
            }
        }
    } else {
        // ---- epilogue warps 2..9: TMEM lane quarter = warp % 4, two warps
        // per quarter (alternate column chunks)
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        uint32_t t = 0;
        ItemView nx = view_item(args, blockIdx.x);
        for (int it = blockIdx.x; it < args.n_items && !abort_flag; it += gridDim.x) {
            const ItemView cur = nx;
            nx = view_item(args, it + gridDim.x);
            const TcItem item = cur.item;
            if (!cur.active) continue;
            const Prob pr = cur.pr;
            const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
            ++t;
            if (!mbar_wait(&acc_full[b], tph, kWaitLimitNs)) {
                if (lane == 0) record_error(args.error, 4u);
                abort_flag = 1;
                break;
            }
            tc_fence_after();
            ws_epilogue(args, item, pr, tmem + b * 128u, quarter, half, lane);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kWsTmemCols);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace

int encode_bucket_map(CUtensorMap* map, const float* base, int n_pad, int count, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return set_error(RSATB_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[3] = {cuuint64_t(n_pad), cuuint64_t(n_pad), cuuint64_t(count)};
    const cuuint64_t strides[2] = {cuuint64_t(n_pad) * 4, cuuint64_t(n_pad) * n_pad * 4};
    const cuuint32_t box[3] = {32u, cuuint32_t(box_rows), 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(RSATB_CUDA_ERROR,
                         "cuTensorMapEncodeTiled failed (%d) for n_pad %d, count %d, box %d",
                         int(r), n_pad, count, box_rows);
    return RSATB_SUCCESS;
}

bool default_tc_ws() {
    const char* s = std::getenv("RSATB_NS_TC");
    return !(s && s[0] == 's');  // "simple": the single-role kernel
}

int prepare_tc_gemm() {
    if (!encode_fn()) return set_error(RSATB_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
    RSATB_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kSmemBytes));
    RSATB_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_ws_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kWsSmemBytes));
    return RSATB_SUCCESS;
}

int launch_tc_gemm(rsatb_context* ctx, const TcMaps& maps, const TcArgs& args, bool ws) {
    if (args.n_items <= 0) return RSATB_SUCCESS;
    int grid = ctx->sm_count;
    if (args.n_items < grid) grid = args.n_items;
    if (ws)
        tc_gemm_ws_kernel<<<grid, 320, kWsSmemBytes, ctx->stream>>>(maps, args);
    else
        tc_gemm_kernel<<<grid, 128, kSmemBytes, ctx->stream>>>(maps, args);
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

}  // namespace ns
}  // namespace rsatb_b200
