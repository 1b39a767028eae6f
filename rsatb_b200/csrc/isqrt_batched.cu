// Batched dense inverse square root by Newton-Schulz: the per-subgraph
// S^-1/2 action of rsatb's graph-local factor (rsatb/calc/isqrtm.hpp:
// 149-232, rsatb/calc/isqrt_action.hpp:1343-1422) for all subgraphs at once,
// with the iteration and stopping rules of rsatb::calc::inverse_sqrt
// (rsatb/calc/isqrtm.hpp:620-807) applied per problem.
//
// Iteration (one step, every GEMM of the form C = A B^T over row-major
// operands, so both tensor-core operands are K-major):
//     W = Z S^T            (= Z S, S symmetric)
//     X = Z W^T            (= Z S Z^T)  -> ||X - I||_F, stopping rules
//     P = 1.875 I - 1.25 X + 0.375 X X^T, made exactly symmetric
//     Z' = P Z
// from Z0 = I / sqrt(s), s >= lambda_max the smaller of the Gershgorin bound
// and ||S||_F.  In the tensor-core phase a problem whose ||X - I||_F is at
// least kLift takes the lift polynomial P = 2.5 I - 2.5 X + X X^T instead
// (poly_coef): it raises the small eigenvalues of X by 6.25 per step instead
// of 3.52 and keeps the spectrum in [0, 9/8]; the FP64 phase, which carries
// the reference's stopping semantics, always takes the reference's polynomial.
//
// Phases: an optional tensor-core phase (all four products in TF32 or
// split TF32 on tcgen05 with FP32 accumulation) followed by FP64 iterations
// (FP64 tensor-core GEMMs).  The iteration is equivariant under Z -> Q Z for
// orthogonal Q, so an antisymmetric part of the rounded left factor P would
// leave a rotation that no later step corrects: P is computed on the tiles
// of its upper triangle only and mirrored, so it is exactly symmetric, and
// a symmetric perturbation only moves Z normal to the solution set, which
// the following steps undo.  Z' = P Z takes Z^T as its K-major B operand,
// which the update itself stores (transposed) for the next step.  Each phase of a chunk is one captured
// CUDA graph; a problem that stops early is gated off in every later kernel
// by its `active` flag and its iterate is retired (copied out) at once.
#include "ns_batched.cuh"
#include "umma.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <vector>

namespace rsatb_b200 {
namespace ns {
namespace {

// ------------------------------------------------------------ kernels

// S (row-major, padded, symmetric from the upper triangle of the
// column-major input) in FP64 and, for a tensor-core phase, as TF32 hi/lo.
__global__ void pack_kernel(const Prob* probs, const int64_t* in_off, const double* M,
                            double* s64, float* s_hi, float* s_lo) {
    const Prob pr = probs[blockIdx.x];
    const double* src = M + in_off[blockIdx.x];
    const int np = pr.n_pad, n = pr.n;
    for (int64_t e = threadIdx.x; e < int64_t(np) * np; e += blockDim.x) {
        const int r = int(e / np), c = int(e - int64_t(r) * np);
        double v = 0.0;
        if (r < n && c < n) v = (r <= c) ? src[int64_t(c) * n + r] : src[int64_t(r) * n + c];
        s64[pr.off + e] = v;
        if (s_hi) {
            const float f = float(v);
            const float h = umma::to_tf32(f);
            s_hi[pr.off + e] = h;
            s_lo[pr.off + e] = f - h;
        }
    }
}

// Scale s >= lambda_max, the smaller of two upper bounds, the Gershgorin
// bound max_r sum_c |S_rc| and the Frobenius norm (the tighter s, the fewer
// steps: X0 = S / s has its smallest eigenvalue lambda_min / s), and the
// starting iterate Z0 = I / sqrt(s) in FP64 (and as TF32 hi/lo for a
// tensor-core phase); state reset.
__global__ void init_kernel(const Prob* probs, const double* s64, State* st, float* z_hi,
                            float* z_lo, double* z64, double* scale, int cap) {
    const Prob pr = probs[blockIdx.x];
    const int np = pr.n_pad, n = pr.n;
    __shared__ double red[256], red2[256];
    double m = 0.0, f2 = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        double s = 0.0;
        const double* row = s64 + pr.off + int64_t(r) * np;
        for (int c = 0; c < n; ++c) {
            s += fabs(row[c]);
            f2 += row[c] * row[c];
        }
        m = fmax(m, s);
    }
    red[threadIdx.x] = m;
    red2[threadIdx.x] = f2;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
            red2[threadIdx.x] += red2[threadIdx.x + w];
        }
        __syncthreads();
    }
    const double s = fmin(red[0], sqrt(red2[0]));
    const double z0 = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    for (int64_t e = threadIdx.x; e < int64_t(np) * np; e += blockDim.x) {
        const int r = int(e / np), c = int(e - int64_t(r) * np);
        const double v = (r == c && r < n) ? z0 : 0.0;
        if (z_hi) {
            const float f = float(v);
            const float h = umma::to_tf32(f);
            z_hi[pr.off + e] = h;
            z_lo[pr.off + e] = f - h;
        }
        z64[pr.off + e] = v;
    }
    if (threadIdx.x == 0) {
        scale[blockIdx.x] = s;
        State x;
        x.norm = 0.0;
        x.norm_pre = 0.0;
        x.count = 0;
        x.active = (s > 0.0 && isfinite(s)) ? 1 : 0;
        x.retire = 0;
        x.status = x.active ? RSATB_SUCCESS : RSATB_NOT_POSITIVE_DEFINITE;
        x.cap = cap;
        x.restart = 0;
        x.lift = 0;
        st[blockIdx.x] = x;
    }
}

// Re-arms the problems for the FP64 phase.  A problem the tensor-core
// phase left far from convergence (diverged, or stopped with ||X - I||_F
// above restart_above: a spectrum the low precision cannot resolve) starts
// over from Z0 in FP64 with the cap restart_cap; the others refine the
// tensor-core iterate with the cap `cap`.  Problems not re-armed are marked
// for the output copy of their last iterate.  The tensor-core phase's
// update count is kept in low_count.
__global__ void rearm_kernel(int np_count, State* st, int* low_count, int from_low, int cap,
                             int restart_cap, double restart_above) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np_count) return;
    State x = st[p];
    low_count[p] = x.count;
    x.restart = 0;
    x.cap = cap;
    if (from_low && (x.status == RSATB_DIVERGED ||
                     (x.status == RSATB_SUCCESS && !(x.norm <= restart_above)))) {
        x.status = RSATB_SUCCESS;
        x.restart = 1;
        x.cap = restart_cap;
    }
    x.active = (x.status == RSATB_SUCCESS) ? 1 : 0;
    x.retire = x.active ? 0 : 1;
    x.count = 0;
    x.norm_pre = 0.0;
    x.lift = 0;
    st[p] = x;
}

// Z64 = I / sqrt(s) for the problems the FP64 phase restarts.
__global__ void restart_kernel(const Prob* probs, const State* st, const double* scale,
                               double* z64) {
    if (!st[blockIdx.x].restart) return;
    const Prob pr = probs[blockIdx.x];
    const int np = pr.n_pad;
    const double s = scale[blockIdx.x];
    const double z0 = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    for (int64_t e = threadIdx.x; e < int64_t(np) * np; e += blockDim.x) {
        const int r = int(e / np), c = int(e - int64_t(r) * np);
        z64[pr.off + e] = (r == c && r < pr.n) ? z0 : 0.0;
    }
}

// The loop condition of rsatb/calc/isqrtm.hpp:615-640 for every active
// problem: continue while norm > tol, count < cap and the residual moved
// by more than 0.5 %; a residual above 100 is a divergence.  With
// stop_on_rise (tensor-core phase) a residual that did not fall also stops:
// in exact arithmetic every eigenvalue error of X shrinks each step, so a
// rise means the low-precision floor was reached.
//
// The plateau and rise tests apply once ||X - I||_F < kQuadratic.  The
// reference runs this loop from a seed already near S^-1/2; here it starts
// from Z0 = I / sqrt(s), where every eigenvalue x of X in (0, 1] climbs
// monotonically (x -> x p(x)^2, about 3.5 x while x is small) and a
// near-null cluster (the gapped spectra of LCAO overlaps) holds the
// Frobenius norm almost still for several steps: a stall of the norm there
// is not a stall of the iteration.
//
// With lift (tensor-core phase) the next P of a problem whose residual is at
// least kLift is the lift polynomial.  Measured on the eigenvalues of the
// benchmark's spectra (n ~ U[40, 400], kappa ~ [1e2, 1e5]), it cuts the
// n^3-weighted mean of the steps to ||X - I||_F < 1e-4 from 10.2 to 7.8
// (continuous) and from 11.3 to 8.4 (gapped).
//
// With floor_stop (tensor-core phase) a step of the cubic polynomial from
// norm_pre < kFloorFrom that ends above twice its exact-arithmetic bound
// also stops: for |e| < 1/2 an eigenvalue error e of X becomes at most
// 1.25 (5/8) |e|^3, so ||X - I||_F falls to at most 0.78 norm_pre^3, and a
// residual above 1.5625 norm_pre^3 is the rounding floor of the phase.  It
// saves the step the rise test needs to see the floor.
constexpr double kQuadratic = 0.5;
constexpr double kLift = 1.0;
constexpr double kFloorFrom = 0.1;
__global__ void control_kernel(int np_count, State* st, double* res2, double tol,
                               int stop_on_rise, int lift, int floor_stop, int* live) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np_count) return;
    State x = st[p];
    const int applied_lift = x.lift;  // the polynomial of the step just taken
    x.retire = 0;
    x.lift = 0;
    if (x.active) {
        const double norm = sqrt(res2[p]);
        x.norm = norm;
        const bool near = norm < kQuadratic;
        bool go = norm > tol && x.count < x.cap &&
                  (!near || fabs(x.norm_pre - norm) > 0.005 * norm);
        if (near && stop_on_rise && x.count > 0 && norm >= x.norm_pre) go = false;
        if (floor_stop && x.count > 0 && !applied_lift && x.norm_pre < kFloorFrom &&
            norm > 1.5625 * x.norm_pre * x.norm_pre * x.norm_pre)
            go = false;
        if (!(norm <= 100.0)) {  // also catches NaN
            x.active = 0;
            x.retire = 1;
            x.status = RSATB_DIVERGED;
        } else if (!go) {
            x.active = 0;
            x.retire = 1;
        } else {
            x.norm_pre = norm;
            x.count += 1;
            x.lift = (lift && norm >= kLift) ? 1 : 0;
            *live = 1;  // every writer stores the same value
        }
    }
    res2[p] = 0.0;
    st[p] = x;
}

// The FP64 phase starts from z64[0]: a problem the tensor-core phase
// stopped while its iterate sat in z64[1] is copied over.
__global__ void retire_low_kernel(const Prob* probs, const State* st, const double* src,
                                  double* dst) {
    if (!st[blockIdx.x].retire) return;
    const Prob pr = probs[blockIdx.x];
    const int np = pr.n_pad;
    for (int64_t e = threadIdx.x; e < int64_t(np) * np; e += blockDim.x)
        dst[pr.off + e] = src[pr.off + e];
}

// z64 = z_hi + z_lo for every problem: the split-TF32 update keeps the
// iterate as a hi/lo pair only, and a problem's tiles are skipped once it
// stops, so the pair still holds the iterate it stopped at.
__global__ void low_to_f64_kernel(const Prob* probs, const float* z_hi, const float* z_lo,
                                  double* z64) {
    const Prob pr = probs[blockIdx.x];
    const int np = pr.n_pad;
    for (int64_t e = threadIdx.x; e < int64_t(np) * np; e += blockDim.x)
        z64[pr.off + e] = double(z_hi[pr.off + e]) + double(z_lo[pr.off + e]);
}

// Result of a problem the FP64 phase just stopped: columns
// [col_start, col_start + k) of (Z + Z^T)/2, column-major n x k.
__global__ void retire_out_kernel(const Prob* probs, const State* st, const double* z64,
                                  const int* col_start, const int* k_cols, const int64_t* out_off,
                                  double* out) {
    if (!st[blockIdx.x].retire) return;
    const Prob pr = probs[blockIdx.x];
    const int np = pr.n_pad, n = pr.n, c0 = col_start[blockIdx.x], k = k_cols[blockIdx.x];
    double* dst = out + out_off[blockIdx.x];
    for (int64_t e = threadIdx.x; e < int64_t(n) * k; e += blockDim.x) {
        const int j = int(e / n), i = int(e - int64_t(j) * n);
        const int c = c0 + j;
        dst[e] = 0.5 * (z64[pr.off + int64_t(i) * np + c] + z64[pr.off + int64_t(c) * np + i]);
    }
}

struct F64Item {
    int p, m0, n0;
};

// D (+)= A B for one m8n8k4 FP64 tile on the tensor cores (mma.sync, the
// FP64 tensor path of sm_100): A 8x4 row-major, one value per lane at
// (lane / 4, lane % 4); B 4x8, one value per lane at (lane % 4, lane / 4);
// D 8x8, two values per lane at (lane / 4, 2 (lane % 4) + {0, 1}).
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// 16 bytes global -> shared, zero-filled when !valid (no bytes read then).
__device__ __forceinline__ void cp16_zfill(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(valid ? 16 : 0)
                 : "memory");
}

// Shared-memory shape of the FP64 GEMM: K chunk KC, [row][k] stride LDR,
// [k][col] stride LDK (both 4 mod 16 doubles: the 16 lanes of a half-warp
// fragment load hit 16 different banks), two stages.
template <bool BT, bool SYM_A>
struct F64Shape {
    static constexpr int KC = SYM_A ? 16 : 32;
    static constexpr int LDR = KC + 4;
    static constexpr int LDK = 64 + 4;
    static constexpr int A_ELEMS = 64 * LDR;
    static constexpr int AT_ELEMS = SYM_A ? KC * LDK : 0;
    static constexpr int B_ELEMS = BT ? 64 * LDR : KC * LDK;
    static constexpr int STAGE = A_ELEMS + AT_ELEMS + B_ELEMS;
    static constexpr size_t SMEM = 2 * size_t(STAGE) * sizeof(double);
};

// FP64 C = A B^T (BT) or C = A B, one 64 x 64 tile per work item, on the
// FP64 tensor cores: 4 warps, each a 32 x 32 quadrant of 4 x 4 m8n8k4
// fragments, K chunks of KC double-buffered in shared memory by cp.async
// (the next chunk is in flight while the current one is multiplied).
// Operands keep the layout their global rows have, so every copy is
// coalesced: rows of A (and of B when BT) as [m][k], rows of B (not BT) and
// of A^T (SYM_A) as [k][n].  SYM_A multiplies by (A + A^T)/2 instead of A,
// summed as the fragment is read.  Same epilogue modes as the tensor-core
// kernel; c_hi/c_lo (optional) receive the TF32 hi/lo split of C for the
// next tensor-core GEMMs.  sym: the items are the tiles on or above the
// diagonal and every element (r, c >= r) is also stored at (c, r), so C
// leaves exactly symmetric (X = Z S Z^T and P, as the reference mirrors
// them, rsatb/calc/isqrtm.hpp:646-669).
template <bool BT, bool SYM_A>
__global__ void __launch_bounds__(128) gemm_f64_kernel(const Prob* probs, const F64Item* items,
                                                       int n_items, const State* st,
                                                       const double* A, const double* B,
                                                       double* C, int mode, const double* Xe,
                                                       double* res2, float* c_hi,
                                                       float* c_lo, int sym, const int* live) {
    if (live && *live == 0) return;  // every problem has stopped
    using Sh = F64Shape<BT, SYM_A>;
    constexpr int KC = Sh::KC, LDR = Sh::LDR, LDK = Sh::LDK;
    extern __shared__ __align__(16) double f64_smem[];
    __shared__ double red[4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int fr = lane >> 2, fc = lane & 3;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const F64Item item = items[it];
        if (!st[item.p].active) continue;
        const Prob pr = probs[item.p];
        const int np = pr.n_pad;
        const double* Ap = A + pr.off;
        const double* Bp = B + pr.off;
        // Copies of chunk k0 into stage s: [64 x KC] row chunks as KC / 2
        // 16-byte units per row, [KC x 64] column chunks as 32 units per k row.
        auto issue = [&](int k0, int s) {
            double* As = f64_smem + s * Sh::STAGE;
            double* AsT = As + Sh::A_ELEMS;
            double* Bs = AsT + Sh::AT_ELEMS;
#pragma unroll
            for (int q = 0; q < KC / 4; ++q) {
                const int idx = threadIdx.x + 128 * q;
                const int r = idx / (KC / 2), u = idx % (KC / 2);
                const int m = item.m0 + r;
                cp16_zfill(As + r * LDR + 2 * u, Ap + (m < np ? int64_t(m) * np + k0 + 2 * u : 0),
                           m < np);
                if (BT) {
                    const int nn = item.n0 + r;
                    cp16_zfill(Bs + r * LDR + 2 * u,
                               Bp + (nn < np ? int64_t(nn) * np + k0 + 2 * u : 0), nn < np);
                }
            }
            if (!BT || SYM_A) {
#pragma unroll
                for (int q = 0; q < KC / 4; ++q) {
                    const int idx = threadIdx.x + 128 * q;
                    const int kr = idx >> 5, u = idx & 31;
                    if (!BT) {
                        const int nn = item.n0 + 2 * u;
                        cp16_zfill(Bs + kr * LDK + 2 * u,
                                   Bp + (nn < np ? int64_t(k0 + kr) * np + nn : 0), nn < np);
                    }
                    if (SYM_A) {
                        const int m = item.m0 + 2 * u;
                        cp16_zfill(AsT + kr * LDK + 2 * u,
                                   Ap + (m < np ? int64_t(k0 + kr) * np + m : 0), m < np);
                    }
                }
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        };
        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
        issue(0, 0);
        for (int k0 = 0, s = 0; k0 < np; k0 += KC, s ^= 1) {
            if (k0 + KC < np) {
                issue(k0 + KC, s ^ 1);
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            }
            __syncthreads();
            const double* As = f64_smem + s * Sh::STAGE;
            const double* AsT = As + Sh::A_ELEMS;
            const double* Bs = AsT + Sh::AT_ELEMS;
#pragma unroll
            for (int kk = 0; kk < KC; kk += 4) {
                double af[4], bf[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int m = wm + 8 * i + fr, k = kk + fc;
                    af[i] = SYM_A ? 0.5 * (As[m * LDR + k] + AsT[k * LDK + m]) : As[m * LDR + k];
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int nn = wn + 8 * j + fr, k = kk + fc;
                    bf[j] = BT ? Bs[nn * LDR + k] : Bs[k * LDK + nn];
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], af[i], bf[j]);
            }
            __syncthreads();  // stage s is refilled by the next iteration's copies
        }
        double r2 = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int m = item.m0 + wm + 8 * i + fr;
            if (m >= np) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int nn = item.n0 + wn + 8 * j + 2 * fc + h;
                    if (nn >= np || (sym && nn < m)) continue;
                    const bool valid = m < pr.n && nn < pr.n;
                    const bool mirror = sym && nn != m;
                    const int64_t e = pr.off + int64_t(m) * np + nn;
                    const int64_t et = pr.off + int64_t(nn) * np + m;
                    double x = acc[i][j][h];
                    if (mode == EPI_POLY)
                        x = fma(0.375, x, fma(-1.25, Xe[e], m == nn ? 1.875 : 0.0));
                    if (!valid) x = 0.0;
                    if (mode == EPI_RESID && valid) {
                        const double d = x - (m == nn ? 1.0 : 0.0);
                        r2 += mirror ? 2.0 * d * d : d * d;
                    }
                    C[e] = x;
                    if (mirror) C[et] = x;
                    if (c_hi) {
                        const float f = float(x);
                        const float hv = umma::to_tf32(f);
                        c_hi[e] = hv;
                        c_lo[e] = f - hv;
                        if (mirror) {
                            c_hi[et] = hv;
                            c_lo[et] = f - hv;
                        }
                    }
                }
            }
        }
        if (mode == EPI_RESID) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            if (lane == 0) red[warp] = r2;
            __syncthreads();
            if (threadIdx.x == 0) {
                const double s = (red[0] + red[1]) + (red[2] + red[3]);
                if (s != 0.0) atomicAdd(res2 + item.p, s);
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------ host side

int ceil_div(int a, int b) { return (a + b - 1) / b; }
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

struct Bucket {
    int n_pad;
    int first;   // first problem (chunk-local index)
    int count;
    int64_t off; // element offset of its first problem
    int nt;      // N tile of the tensor-core GEMM
};

// Workspace of one chunk, carved from the context scratch.
struct Chunk {
    std::vector<int> ids;  // caller's problem index of each chunk-local problem
    std::vector<Prob> probs;
    std::vector<Bucket> buckets;
    int64_t elems = 0;     // sum of n_pad^2
};

struct Arrays {
    // tensor-core phase (nullptr when absent); zt: Z^T, the B operand of the
    // split-TF32 update Z' = P Z (two buffers: one read, one written)
    float *s_hi, *s_lo, *z_hi, *z_lo, *w_hi, *w_lo, *x_hi, *x_lo,
        *p_hi, *p_lo, *zt_hi[2], *zt_lo[2];
    // FP64 phase
    double *s64, *z64[2], *w64, *x64, *p64;
};

size_t chunk_bytes(int64_t elems, bool low) {
    return size_t(elems) * ((low ? 14 * 4 : 0) + 6 * 8);
}

// The tensor-core phase's update Z' = P Z: split TF32 on the tensor cores
// with P made exactly symmetric (the default), or in FP64 with (P + P^T)/2
// summed as it is read (RSATB_NS_UPDATE=fp64).
bool fp64_update() {
    const char* s = std::getenv("RSATB_NS_UPDATE");
    return s && s[0] == 'f';
}

// The lift polynomial in the tensor-core phase (the default), or the
// reference's polynomial throughout (RSATB_NS_LIFT=0).
bool lift_enabled() {
    const char* s = std::getenv("RSATB_NS_LIFT");
    return !(s && s[0] == '0');
}

// The floor test of the tensor-core phase (the default; RSATB_NS_FLOOR=0:
// the plateau and rise tests only).
bool floor_stop_enabled() {
    const char* s = std::getenv("RSATB_NS_FLOOR");
    return !(s && s[0] == '0');
}

// A tensor-core phase that stops above this residual has not resolved the
// spectrum; the FP64 phase starts that problem over from Z0.
constexpr double kRestartAbove = 0.25;

struct Opts {
    int precision;
    int max_iter;
    int max_fp64;
    int max_fp64_restart;
    double tol;
    double accept;
    size_t workspace;
    bool graph;
    bool ws;                                // warp-specialised tensor-core kernel
    std::vector<std::pair<int, int>> tiles; // (n_pad, N tile) overrides
};

// Device views of one chunk's tables and arrays.
struct Dev {
    Prob* probs;
    int64_t* in_off;
    int64_t* out_off;
    int* col_start;
    int* k_cols;
    State* state;
    double* res2;
    double* scale;
    int* low_count;
    unsigned* error;
    TcItem* tc_items;
    TcItem* tc_items_upper;  // the tiles that touch the upper triangle
    F64Item* f64_items;
    F64Item* f64_items_upper;  // the 64 x 64 tiles on or above the diagonal
    // live[k] (tensor-core phase) and live_f64[k] (FP64 phase): set by the
    // control step of iteration k when a problem goes on; the GEMMs after it
    // return at once when it stays 0 (the graph keeps the full loop).
    int* live;
    int* live_f64;
    int n_live;
    int n_tc_items;
    int n_f64_items;
    int n_f64_upper;
    Arrays a;
};

template <typename T>
T* carve(char*& cur, size_t count) {
    T* p = reinterpret_cast<T*>(cur);
    cur += align256(count * sizeof(T));
    return p;
}

// One tensor-core GEMM over the whole chunk, in launches of at most
// kMaxBuckets buckets.
// items / group_item_begin: the full tile list or the upper-triangle one
// (sym); ct_hi / ct_lo: optional transposed store of C.
int tc_gemm(rsatb_context* ctx, const Chunk& ch, const Dev& d, const TcItem* items,
            const std::vector<int>& group_item_begin, const float* a_hi, const float* a_lo,
            const float* b_hi, const float* b_lo, float* c_hi, float* c_lo, double* c64,
            int mode, const float* xe_hi, const float* xe_lo, bool split, bool ws,
            rsatb_isqrt_stats* stats, float* ct_hi = nullptr, float* ct_lo = nullptr,
            bool sym = false, const int* live = nullptr) {
    const int nb = int(ch.buckets.size());
    for (int g0 = 0, gi = 0; g0 < nb; g0 += kMaxBuckets, ++gi) {
        TcMaps maps;
        for (int b = g0; b < std::min(nb, g0 + kMaxBuckets); ++b) {
            const Bucket& bk = ch.buckets[b];
            const int lb = b - g0;
            RSATB_TRY(encode_bucket_map(&maps.a_hi[lb], a_hi + bk.off, bk.n_pad, bk.count, 128));
            RSATB_TRY(encode_bucket_map(&maps.a_lo[lb], a_lo + bk.off, bk.n_pad, bk.count, 128));
            RSATB_TRY(encode_bucket_map(&maps.b_hi[lb], b_hi + bk.off, bk.n_pad, bk.count, bk.nt));
            RSATB_TRY(encode_bucket_map(&maps.b_lo[lb], b_lo + bk.off, bk.n_pad, bk.count, bk.nt));
        }
        TcArgs args{};
        args.probs = d.probs;
        args.items = items + group_item_begin[gi];
        args.n_items = group_item_begin[gi + 1] - group_item_begin[gi];
        args.state = d.state;
        args.c_hi = c_hi;
        args.c_lo = c_lo;
        args.c64 = c64;
        args.xe_hi = xe_hi;
        args.xe_lo = xe_lo;
        args.res2 = d.res2;
        args.mode = mode;
        args.ct_hi = ct_hi;
        args.ct_lo = ct_lo;
        args.sym = sym ? 1 : 0;
        args.split = split ? 1 : 0;
        args.error = d.error;
        args.live = live;
        RSATB_TRY(launch_tc_gemm(ctx, maps, args, ws));
        if (stats) stats->gemm_launches++;
    }
    return RSATB_SUCCESS;
}

// sym: C is symmetric (X, P); only the tiles on or above the diagonal are
// computed, each mirrored.
template <bool BT, bool SYM_A = false>
int f64_gemm(rsatb_context* ctx, const Dev& d, const double* A, const double* B, double* C,
             int mode, const double* Xe, rsatb_isqrt_stats* stats, float* c_hi = nullptr,
             float* c_lo = nullptr, bool sym = false, const int* live = nullptr) {
    const F64Item* items = sym ? d.f64_items_upper : d.f64_items;
    const int n_items = sym ? d.n_f64_upper : d.n_f64_items;
    if (n_items == 0) return RSATB_SUCCESS;
    int grid = ctx->sm_count * 6;
    if (n_items < grid) grid = n_items;
    gemm_f64_kernel<BT, SYM_A><<<grid, 128, F64Shape<BT, SYM_A>::SMEM, ctx->stream>>>(
        d.probs, items, n_items, d.state, A, B, C, mode, Xe, d.res2, c_hi, c_lo, sym ? 1 : 0,
        live);
    RSATB_LAUNCH_CHECK(ctx);
    if (stats) stats->gemm_launches++;
    return RSATB_SUCCESS;
}

// Issues `body` either directly or as one captured graph on the context's
// stream.
template <typename F>
int run_phase(rsatb_context* ctx, bool graph, F&& body) {
    if (!graph || ctx->stream == nullptr) return body();
    RSATB_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int st = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (st != RSATB_SUCCESS) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "graph capture failed: %s", cudaGetErrorString(e));
    cudaGraphExec_t x = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "graph instantiation failed: %s",
                         cudaGetErrorString(ie));
    const cudaError_t le = cudaGraphLaunch(x, ctx->stream);
    const cudaError_t se = cudaStreamSynchronize(ctx->stream);
    cudaGraphExecDestroy(x);
    if (le != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "graph launch failed: %s", cudaGetErrorString(le));
    if (se != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "graph run failed: %s", cudaGetErrorString(se));
    return RSATB_SUCCESS;
}

int run_chunk(rsatb_context* ctx, const Opts& o, const Chunk& ch, const int* col_start_h,
              const int* k_cols_h, const int64_t* in_off_h, const int64_t* out_off_h,
              const double* M, double* out, std::vector<State>& st_out,
              std::vector<int>& low_count_out, rsatb_isqrt_stats* stats) {
    const int P = int(ch.probs.size());
    const bool low = o.precision != RSATB_NS_FP64;
    const bool split = o.precision == RSATB_NS_TF32X3;
    // Dynamic shared-memory opt-in of the FP64 GEMMs, before any capture.
    RSATB_CUDA_TRY(cudaFuncSetAttribute(gemm_f64_kernel<true, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(F64Shape<true, false>::SMEM)));
    RSATB_CUDA_TRY(cudaFuncSetAttribute(gemm_f64_kernel<false, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(F64Shape<false, true>::SMEM)));
    RSATB_CUDA_TRY(cudaFuncSetAttribute(gemm_f64_kernel<false, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(F64Shape<false, false>::SMEM)));

    // Work items, ordered by bucket (the buckets of a launch group are
    // contiguous), largest problems first.
    std::vector<TcItem> tc_items, tc_upper;
    std::vector<int> group_begin{0}, group_begin_upper{0};
    std::vector<F64Item> f64_items, f64_upper;
    for (size_t b = 0; b < ch.buckets.size(); ++b) {
        const Bucket& bk = ch.buckets[b];
        for (int z = 0; z < bk.count; ++z) {
            const int p = bk.first + z;
            if (low)
                for (int m0 = 0; m0 < bk.n_pad; m0 += 128)
                    for (int n0 = 0; n0 < bk.n_pad; n0 += bk.nt) {
                        const TcItem it{p, int(b % kMaxBuckets), z, m0, n0, bk.nt};
                        tc_items.push_back(it);
                        if (n0 + bk.nt > m0) tc_upper.push_back(it);  // reaches col >= row
                    }
            for (int m0 = 0; m0 < bk.n_pad; m0 += 64)
                for (int n0 = 0; n0 < bk.n_pad; n0 += 64) {
                    f64_items.push_back(F64Item{p, m0, n0});
                    if (n0 >= m0) f64_upper.push_back(F64Item{p, m0, n0});
                }
        }
        if ((b + 1) % kMaxBuckets == 0 || b + 1 == ch.buckets.size()) {
            group_begin.push_back(int(tc_items.size()));
            group_begin_upper.push_back(int(tc_upper.size()));
        }
    }

    // Workspace.
    const int64_t E = ch.elems;
    size_t bytes = 0;
    bytes += align256(P * sizeof(Prob)) + 2 * align256(P * sizeof(int64_t)) +
             3 * align256(P * sizeof(int)) + align256(P * sizeof(State)) +
             2 * align256(P * sizeof(double)) + 256 +
             align256(tc_items.size() * sizeof(TcItem)) +
             align256(tc_upper.size() * sizeof(TcItem)) +
             align256(f64_items.size() * sizeof(F64Item)) +
             align256(f64_upper.size() * sizeof(F64Item)) +
             align256(size_t(o.max_iter + 2 + std::max(o.max_fp64, o.max_fp64_restart) + 2) *
                      sizeof(int));
    bytes += (low ? 14 * align256(E * sizeof(float)) : 0) + 6 * align256(E * sizeof(double));
    void* ws = nullptr;
    RSATB_TRY(ctx_scratch(ctx, bytes, &ws));
    char* cur = static_cast<char*>(ws);
    Dev d{};
    d.probs = carve<Prob>(cur, P);
    d.in_off = carve<int64_t>(cur, P);
    d.out_off = carve<int64_t>(cur, P);
    d.col_start = carve<int>(cur, P);
    d.k_cols = carve<int>(cur, P);
    d.low_count = carve<int>(cur, P);
    d.state = carve<State>(cur, P);
    d.res2 = carve<double>(cur, P);
    d.scale = carve<double>(cur, P);
    d.error = carve<unsigned>(cur, 64);
    d.tc_items = carve<TcItem>(cur, tc_items.size());
    d.tc_items_upper = carve<TcItem>(cur, tc_upper.size());
    d.f64_items = carve<F64Item>(cur, f64_items.size());
    d.f64_items_upper = carve<F64Item>(cur, f64_upper.size());
    d.n_live = o.max_iter + 2 + std::max(o.max_fp64, o.max_fp64_restart) + 2;
    d.live = carve<int>(cur, size_t(d.n_live));
    d.live_f64 = d.live + (o.max_iter + 2);
    d.n_tc_items = int(tc_items.size());
    d.n_f64_items = int(f64_items.size());
    d.n_f64_upper = int(f64_upper.size());
    Arrays& a = d.a;
    a = Arrays{};
    if (low) {
        a.s_hi = carve<float>(cur, E);
        a.s_lo = carve<float>(cur, E);
        a.z_hi = carve<float>(cur, E);
        a.z_lo = carve<float>(cur, E);
        a.w_hi = carve<float>(cur, E);
        a.w_lo = carve<float>(cur, E);
        a.x_hi = carve<float>(cur, E);
        a.x_lo = carve<float>(cur, E);
        a.p_hi = carve<float>(cur, E);
        a.p_lo = carve<float>(cur, E);
        for (int i = 0; i < 2; ++i) {
            a.zt_hi[i] = carve<float>(cur, E);
            a.zt_lo[i] = carve<float>(cur, E);
        }
    }
    a.s64 = carve<double>(cur, E);
    a.z64[0] = carve<double>(cur, E);
    a.z64[1] = carve<double>(cur, E);
    a.w64 = carve<double>(cur, E);
    a.x64 = carve<double>(cur, E);
    a.p64 = carve<double>(cur, E);

    // Tables.
    std::vector<int64_t> in_off(P), out_off(P);
    std::vector<int> cs(P), kc(P);
    for (int i = 0; i < P; ++i) {
        const int id = ch.ids[i];
        in_off[i] = in_off_h[id];
        out_off[i] = out_off_h[id];
        cs[i] = col_start_h ? col_start_h[id] : 0;
        kc[i] = (k_cols_h && k_cols_h[id] > 0) ? k_cols_h[id] : ch.probs[i].n;
    }
    cudaStream_t s = ctx->stream;
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.probs, ch.probs.data(), P * sizeof(Prob),
                                   cudaMemcpyHostToDevice, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.in_off, in_off.data(), P * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.out_off, out_off.data(), P * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.col_start, cs.data(), P * sizeof(int),
                                   cudaMemcpyHostToDevice, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.k_cols, kc.data(), P * sizeof(int),
                                   cudaMemcpyHostToDevice, s));
    if (!tc_items.empty())
        RSATB_CUDA_TRY(cudaMemcpyAsync(d.tc_items, tc_items.data(),
                                       tc_items.size() * sizeof(TcItem), cudaMemcpyHostToDevice,
                                       s));
    if (!tc_upper.empty())
        RSATB_CUDA_TRY(cudaMemcpyAsync(d.tc_items_upper, tc_upper.data(),
                                       tc_upper.size() * sizeof(TcItem), cudaMemcpyHostToDevice,
                                       s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.f64_items, f64_items.data(),
                                   f64_items.size() * sizeof(F64Item), cudaMemcpyHostToDevice, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d.f64_items_upper, f64_upper.data(),
                                   f64_upper.size() * sizeof(F64Item), cudaMemcpyHostToDevice, s));
    RSATB_CUDA_TRY(cudaMemsetAsync(d.res2, 0, P * sizeof(double), s));
    RSATB_CUDA_TRY(cudaMemsetAsync(d.error, 0, sizeof(unsigned), s));
    RSATB_CUDA_TRY(cudaMemsetAsync(d.live, 0, size_t(d.n_live) * sizeof(int), s));

    // Pack S and the starting iterate.
    pack_kernel<<<P, 256, 0, s>>>(d.probs, d.in_off, M, a.s64, a.s_hi, a.s_lo);
    RSATB_LAUNCH_CHECK(ctx);
    init_kernel<<<P, 256, 0, s>>>(d.probs, a.s64, d.state, a.z_hi, a.z_lo, a.z64[0], d.scale,
                                  low ? o.max_iter : o.max_fp64);
    RSATB_LAUNCH_CHECK(ctx);
    if (low) {  // Z0 = I / sqrt(s) is symmetric: Z0^T = Z0
        RSATB_CUDA_TRY(cudaMemcpyAsync(a.zt_hi[0], a.z_hi, E * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s));
        RSATB_CUDA_TRY(cudaMemcpyAsync(a.zt_lo[0], a.z_lo, E * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s));
    }
    const int cb = (P + 255) / 256;

    cudaEvent_t ev[3];
    for (auto& e : ev) RSATB_CUDA_TRY(cudaEventCreate(&e));
    struct EvGuard {
        cudaEvent_t* e;
        ~EvGuard() {
            for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]);
        }
    } guard{ev};
    RSATB_CUDA_TRY(cudaEventRecord(ev[0], s));

    // With the FP64 update P is consumed in FP64 only: the tensor-core
    // kernel that can skip its TF32 hi/lo copy does so.
    const bool use_ws_tc = o.ws;
    const bool update64 = fp64_update();
    const int lift = lift_enabled() ? 1 : 0;
    const int floor_stop = floor_stop_enabled() ? 1 : 0;
    if (low) {
        RSATB_TRY(prepare_tc_gemm());
        RSATB_TRY(run_phase(ctx, o.graph, [&]() -> int {
            for (int k = 0; k <= o.max_iter; ++k) {
                const int c = k & 1;
                const int* live_in = k ? d.live + (k - 1) : nullptr;  // after control k - 1
                const int* live_k = d.live + k;                        // after control k
                // W = Z S^T, X = Z W^T (+ residual) on the tensor cores
                RSATB_TRY(tc_gemm(ctx, ch, d, d.tc_items, group_begin, a.z_hi, a.z_lo, a.s_hi,
                                  a.s_lo, a.w_hi, a.w_lo, nullptr, EPI_STORE, nullptr, nullptr,
                                  split, o.ws, stats, nullptr, nullptr, false, live_in));
                // X on every tile (its upper triangle mirrored, as P is, measured
                // the same: 21,300 against 21,400 matrices/s at 20,000 problems).
                RSATB_TRY(tc_gemm(ctx, ch, d, d.tc_items, group_begin, a.z_hi, a.z_lo, a.w_hi,
                                  a.w_lo, a.x_hi, a.x_lo, nullptr, EPI_RESID, nullptr, nullptr,
                                  split, o.ws, stats, nullptr, nullptr, false, live_in));
                control_kernel<<<cb, 256, 0, s>>>(P, d.state, d.res2, o.tol, 1, lift,
                                                  floor_stop, d.live + k);
                RSATB_LAUNCH_CHECK(ctx);
                if (c == 1 && update64) {
                    retire_low_kernel<<<P, 256, 0, s>>>(d.probs, d.state, a.z64[1], a.z64[0]);
                    RSATB_LAUNCH_CHECK(ctx);
                }
                if (k == o.max_iter) break;
                // P = 1.875 I - 1.25 X + 0.375 X X^T (or the lift polynomial) on
                // the tensor cores, then
                // Z' = P Z with P exactly symmetric.  A symmetric factor on the
                // left only moves Z off the solution set {Q S^-1/2}, which later
                // steps undo; the antisymmetric part of a rounded P would add a
                // rotation Q that no step removes (split TF32 with an
                // unsymmetrised P: 6e-4 from the eigen route at kappa 1e5,
                // symmetrised: 2.4e-5, as with the FP64 update).
                if (!update64) {
                    // Upper-triangle tiles of P, each element also stored
                    // mirrored; Z' = P Z against Z^T (both operands K-major),
                    // storing Z' and Z'^T (the FP64 iterate is formed once,
                    // after the phase).
                    RSATB_TRY(tc_gemm(ctx, ch, d, d.tc_items_upper, group_begin_upper, a.x_hi,
                                      a.x_lo, a.x_hi, a.x_lo, a.p_hi, a.p_lo, nullptr, EPI_POLY,
                                      a.x_hi, a.x_lo, split, o.ws, stats, nullptr, nullptr, true,
                                      live_k));
                    RSATB_TRY(tc_gemm(ctx, ch, d, d.tc_items, group_begin, a.p_hi, a.p_lo,
                                      a.zt_hi[c], a.zt_lo[c], a.z_hi, a.z_lo, nullptr,
                                      EPI_STORE, nullptr, nullptr, split, o.ws, stats,
                                      a.zt_hi[c ^ 1], a.zt_lo[c ^ 1], false, live_k));
                } else {
                    RSATB_TRY(tc_gemm(ctx, ch, d, d.tc_items, group_begin, a.x_hi, a.x_lo, a.x_hi,
                                      a.x_lo, use_ws_tc ? nullptr : a.p_hi,
                                      use_ws_tc ? nullptr : a.p_lo, a.p64, EPI_POLY, a.x_hi,
                                      a.x_lo, split, o.ws, stats, nullptr, nullptr, false,
                                      live_k));
                    const int st_z = f64_gemm<false, true>(ctx, d, a.p64, a.z64[c], a.z64[c ^ 1],
                                                           EPI_STORE, nullptr, stats, a.z_hi,
                                                           a.z_lo, false, live_k);
                    RSATB_TRY(st_z);
                }
            }
            return RSATB_SUCCESS;
        }));
    }
    if (low && !update64) {
        low_to_f64_kernel<<<P, 256, 0, s>>>(d.probs, a.z_hi, a.z_lo, a.z64[0]);
        RSATB_LAUNCH_CHECK(ctx);
    }
    RSATB_CUDA_TRY(cudaEventRecord(ev[1], s));

    rearm_kernel<<<cb, 256, 0, s>>>(P, d.state, d.low_count, low ? 1 : 0, o.max_fp64,
                                    o.max_fp64_restart, kRestartAbove);
    RSATB_LAUNCH_CHECK(ctx);
    restart_kernel<<<P, 256, 0, s>>>(d.probs, d.state, d.scale, a.z64[0]);
    RSATB_LAUNCH_CHECK(ctx);
    retire_out_kernel<<<P, 256, 0, s>>>(d.probs, d.state, a.z64[0], d.col_start, d.k_cols,
                                        d.out_off, out);
    RSATB_LAUNCH_CHECK(ctx);
    int fp64_steps = o.max_fp64;
    if (low) {
        // The FP64 loop is as long as the largest cap among the re-armed
        // problems (a restart needs the full FP64 iteration count).
        std::vector<State> h(P);
        RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), d.state, P * sizeof(State),
                                       cudaMemcpyDeviceToHost, s));
        RSATB_CUDA_TRY(cudaStreamSynchronize(s));
        for (const State& x : h)
            if (x.active && x.cap > fp64_steps) fp64_steps = x.cap;
    }

    RSATB_TRY(run_phase(ctx, o.graph, [&]() -> int {
        for (int k = 0; k <= fp64_steps; ++k) {
            const int c = k & 1;
            const int* live_in = k ? d.live_f64 + (k - 1) : nullptr;
            const int* live_k = d.live_f64 + k;
            RSATB_TRY(f64_gemm<true>(ctx, d, a.z64[c], a.s64, a.w64, EPI_STORE, nullptr, stats,
                                     nullptr, nullptr, false, live_in));
            RSATB_TRY(f64_gemm<true>(ctx, d, a.z64[c], a.w64, a.x64, EPI_RESID, nullptr, stats,
                                     nullptr, nullptr, true, live_in));
            control_kernel<<<cb, 256, 0, s>>>(P, d.state, d.res2, o.tol, 0, 0, 0,
                                              d.live_f64 + k);
            RSATB_LAUNCH_CHECK(ctx);
            retire_out_kernel<<<P, 256, 0, s>>>(d.probs, d.state, a.z64[c], d.col_start,
                                                d.k_cols, d.out_off, out);
            RSATB_LAUNCH_CHECK(ctx);
            if (k == fp64_steps) break;
            // X and P exactly symmetric (upper tiles, mirrored): Z' = P Z
            // takes P as it is.
            RSATB_TRY(f64_gemm<true>(ctx, d, a.x64, a.x64, a.p64, EPI_POLY, a.x64, stats,
                                     nullptr, nullptr, true, live_k));
            const int st_z = f64_gemm<false, false>(ctx, d, a.p64, a.z64[c], a.z64[c ^ 1],
                                                   EPI_STORE, nullptr, stats, nullptr, nullptr,
                                                   false, live_k);
            RSATB_TRY(st_z);
        }
        return RSATB_SUCCESS;
    }));
    RSATB_CUDA_TRY(cudaEventRecord(ev[2], s));

    // Results back.
    st_out.resize(P);
    low_count_out.resize(P);
    unsigned err = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(st_out.data(), d.state, P * sizeof(State),
                                   cudaMemcpyDeviceToHost, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(low_count_out.data(), d.low_count, P * sizeof(int),
                                   cudaMemcpyDeviceToHost, s));
    RSATB_CUDA_TRY(cudaMemcpyAsync(&err, d.error, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    RSATB_CUDA_TRY(cudaStreamSynchronize(s));
    if (err)
        return set_error(RSATB_CUDA_ERROR,
                         "tensor-core GEMM gave up on a bounded wait (code %u): a TMA load or an "
                         "MMA did not complete within 2 s",
                         err);
    if (stats) {
        float t1 = 0.f, t2 = 0.f;
        cudaEventElapsedTime(&t1, ev[0], ev[1]);
        cudaEventElapsedTime(&t2, ev[1], ev[2]);
        stats->low_ms += t1;
        stats->fp64_ms += t2;
        for (int i = 0; i < P; ++i) {
            const double n = ch.probs[i].n, np = ch.probs[i].n_pad;
            const int lc = low ? low_count_out[i] : 0;
            const int fc = st_out[i].count;
            // Tile FLOPs: every pass computes G1, G2; full steps add G3, G4.
            const int bucket_nt = [&] {
                for (const Bucket& b : ch.buckets)
                    if (i >= b.first && i < b.first + b.count) return b.nt;
                return 0;
            }();
            const double tile = 2.0 * ceil_div(int(np), 128) * 128.0 * np *
                                (ceil_div(int(np), bucket_nt ? bucket_nt : 1) * bucket_nt);
            if (low) stats->low_flops += tile * (split ? 3 : 1) * (2.0 * (lc + 1) + 2.0 * lc);
            // FP64 passes: W and X (X on the upper tiles, a share u of them),
            // full steps add P (upper tiles) and Z'.
            const int t64 = ceil_div(int(np), 64);
            const double u = 0.5 * (t64 + 1) / t64;
            stats->fp64_flops += 2.0 * n * n * n * (1.0 + u) * ((fc + 1) + fc);
            stats->useful_flops += 8.0 * n * n * n * (lc + fc);
        }
    }
    return RSATB_SUCCESS;
}

}  // namespace
}  // namespace ns
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_isqrt_columns_batched(rsatb_ctx_t ctx, int n_problems, const int32_t* n,
                                           const int32_t* col_start, const int32_t* k_cols,
                                           const int64_t* in_offset, const double* M,
                                           const int64_t* out_offset, double* out,
                                           const rsatb_isqrt_options* options, int32_t* status,
                                           rsatb_isqrt_stats* stats) {
    using namespace rsatb_b200::ns;
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (n_problems < 0) return set_error(RSATB_INVALID_ARGUMENT, "n_problems < 0");
    if (stats) *stats = rsatb_isqrt_stats{};
    if (n_problems == 0) return RSATB_SUCCESS;
    if (!n || !in_offset || !out_offset || !M || !out)
        return set_error(RSATB_INVALID_ARGUMENT, "null argument");
    Opts o{};
    o.precision = options ? options->precision : RSATB_NS_FP64;
    if (o.precision < RSATB_NS_FP64 || o.precision > RSATB_NS_TF32)
        return set_error(RSATB_INVALID_ARGUMENT, "unknown precision %d", o.precision);
    const bool low = o.precision != RSATB_NS_FP64;
    o.max_iter = (options && options->max_iter > 0) ? options->max_iter : 30;
    o.max_fp64 = (options && options->max_fp64_iter > 0) ? options->max_fp64_iter
                                                          : (low ? 6 : 60);
    o.max_fp64_restart = std::max(o.max_fp64, 60);
    o.tol = (options && options->tol > 0) ? options->tol : 1e-11;
    o.accept = (options && options->accept > 0) ? options->accept : 1e-6;
    o.workspace = (options && options->workspace_bytes) ? options->workspace_bytes
                                                        : (size_t(8) << 30);
    o.graph = !(options && options->no_graph);
    const int tck = options ? options->tc_kernel : 0;
    if (tck < 0 || tck > 2) return set_error(RSATB_INVALID_ARGUMENT, "unknown tc_kernel %d", tck);
    o.ws = tck == 0 ? default_tc_ws() : tck == 1;
    if (options && options->n_tiles > 0) {
        if (!options->tile_n_pad || !options->tile_nt)
            return set_error(RSATB_INVALID_ARGUMENT, "n_tiles > 0 with a null tile table");
        for (int t = 0; t < options->n_tiles; ++t) {
            const int np = options->tile_n_pad[t], nt = options->tile_nt[t];
            if (np < 32 || np % 32 || nt < 16 || nt % 16 || nt > tc_max_nt(o.ws))
                return set_error(RSATB_INVALID_ARGUMENT,
                                 "tile %d: n_pad %d / N tile %d (N tile a multiple of 16 up to "
                                 "%d, n_pad a multiple of 32)",
                                 t, np, nt, tc_max_nt(o.ws));
            o.tiles.emplace_back(np, nt);
        }
    }
    for (int p = 0; p < n_problems; ++p) {
        if (n[p] < 1 || n[p] > 1024)
            return set_error(RSATB_INVALID_ARGUMENT, "problem %d: n = %d outside [1, 1024]", p,
                             n[p]);
        const int c0 = col_start ? col_start[p] : 0;
        const int k = (k_cols && k_cols[p] > 0) ? k_cols[p] : n[p];
        if (c0 < 0 || c0 + k > n[p])
            return set_error(RSATB_INVALID_ARGUMENT,
                             "problem %d: columns [%d, %d) outside the %d x %d matrix", p, c0,
                             c0 + k, n[p], n[p]);
        if (in_offset[p] < 0 || out_offset[p] < 0)
            return set_error(RSATB_INVALID_ARGUMENT, "problem %d: negative offset", p);
    }
    if (!(reinterpret_cast<uintptr_t>(M) % 8 == 0) || !(reinterpret_cast<uintptr_t>(out) % 8 == 0))
        return set_error(RSATB_INVALID_ARGUMENT, "M and out must be 8-byte aligned");

    // Graph capture needs a capturable stream: on the legacy default stream
    // the call runs on the context's own stream, ordered after the work
    // already queued on the caller's.
    struct StreamSwap {
        rsatb_context* ctx;
        cudaStream_t saved;
        ~StreamSwap() { ctx->stream = saved; }
    } swap{ctx, ctx->stream};
    if (o.graph && ctx->stream == nullptr && ctx->own_stream != nullptr) {
        cudaEvent_t e;
        RSATB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        cudaError_t r1 = cudaEventRecord(e, nullptr);
        cudaError_t r2 = cudaStreamWaitEvent(ctx->own_stream, e, 0);
        cudaEventDestroy(e);
        RSATB_CUDA_TRY(r1);
        RSATB_CUDA_TRY(r2);
        ctx->stream = ctx->own_stream;
    }

    // Largest first, so each chunk's buckets are ordered and the persistent
    // CTAs start on the longest tiles.
    std::vector<int> order(n_problems);
    std::iota(order.begin(), order.end(), 0);
    auto npad = [&](int p) { return (n[p] + 31) / 32 * 32; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return npad(x) > npad(y); });

    std::vector<State> st;
    std::vector<int> lc;
    size_t pos = 0;
    while (pos < order.size()) {
        Chunk ch;
        int64_t elems = 0;
        while (pos < order.size()) {
            const int p = order[pos];
            const int64_t e = int64_t(npad(p)) * npad(p);
            if (!ch.ids.empty() && chunk_bytes(elems + e, low) > o.workspace) break;
            const int np = npad(p);
            if (ch.buckets.empty() || ch.buckets.back().n_pad != np) {
                const int max_nt = low ? tc_max_nt(o.ws) : 256;
                const int tiles = (np + max_nt - 1) / max_nt;
                int nt = ((np + tiles - 1) / tiles + 15) / 16 * 16;
                for (const auto& t : o.tiles)
                    if (t.first == np) nt = t.second;
                ch.buckets.push_back(Bucket{np, int(ch.ids.size()), 0, elems, nt});
            }
            ch.buckets.back().count++;
            ch.ids.push_back(p);
            ch.probs.push_back(Prob{n[p], np, elems});
            elems += e;
            ++pos;
        }
        ch.elems = elems;
        RSATB_TRY(run_chunk(ctx, o, ch, col_start, k_cols, in_offset, out_offset, M, out, st, lc,
                            stats));
        for (size_t i = 0; i < ch.ids.size(); ++i) {
            const State& x = st[i];
            int s = x.status;
            if (s == RSATB_SUCCESS && !(x.norm <= o.accept)) s = RSATB_NUMERICAL_FAILURE;
            if (status) status[ch.ids[i]] = s;
            if (stats) {
                stats->low_iterations = std::max(stats->low_iterations, lc[i]);
                stats->fp64_iterations = std::max(stats->fp64_iterations, x.count);
                if (s != RSATB_SUCCESS) stats->n_failed++;
                if (std::isfinite(x.norm))
                    stats->max_residual = std::max(stats->max_residual, x.norm);
                else
                    stats->max_residual = INFINITY;
            }
        }
        if (stats) stats->chunks++;
    }
    return RSATB_SUCCESS;
}

// ------------------------------------------------------------- autotuner

namespace rsatb_b200 {
namespace ns {
namespace {

// count column-major n x n matrices M_p = I + (0.5 / n) H_p with H_p
// symmetric, zero diagonal, entries uniform in [-1, 1) from a counter hash
// (splitmix64 finaliser of (seed, p, min(i, j), max(i, j))): by Gershgorin
// the spectrum lies in [0.5, 1.5], so every sample is SPD.
__global__ void spd_sample_kernel(double* M, int n, int count, uint64_t seed) {
    const int64_t nn = int64_t(n) * n;
    const int64_t total = nn * count;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t p = e / nn;
        const int rem = int(e - p * nn);
        const int i = rem % n, j = rem / n;
        double v = 1.0;
        if (i != j) {
            uint64_t x = seed ^ (uint64_t(p) * 0x9E3779B97F4A7C15ull) ^
                         (uint64_t(min(i, j)) << 32) ^ uint64_t(max(i, j));
            x ^= x >> 30;
            x *= 0xBF58476D1CE4E5B9ull;
            x ^= x >> 27;
            x *= 0x94D049BB133111EBull;
            x ^= x >> 31;
            const double uni = double(x >> 11) * (1.0 / 9007199254740992.0);
            v = (0.5 / n) * (2.0 * uni - 1.0);
        }
        M[e] = v;
    }
}

// N tile of candidate `idx` (caps 32, 64, 128, 256 columns) for a padded
// size, 0 when the kernel does not take it or an earlier cap gives the same.
int candidate_nt(int np, bool ws, int idx) {
    static const int caps[4] = {32, 64, 128, 256};
    auto rule = [&](int cap) {
        const int tiles = (np + cap - 1) / cap;
        return ((np + tiles - 1) / tiles + 15) / 16 * 16;
    };
    if (caps[idx] > tc_max_nt(ws)) return 0;
    const int nt = rule(caps[idx]);
    for (int k = 0; k < idx; ++k)
        if (rule(caps[k]) == nt) return 0;
    return nt;
}

}  // namespace
}  // namespace ns
}  // namespace rsatb_b200

extern "C" int rsatb_isqrt_autotune(rsatb_ctx_t ctx, int precision, int n_sizes,
                                   const int32_t* sizes, int problems_per_size,
                                   int* tc_kernel_out, int32_t* nt_out, double* ms_out) {
    using namespace rsatb_b200::ns;
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (precision != RSATB_NS_TF32X3 && precision != RSATB_NS_TF32)
        return set_error(RSATB_INVALID_ARGUMENT,
                         "autotuning needs a tensor-core precision (RSATB_NS_TF32X3 or TF32)");
    if (n_sizes < 1 || !sizes || !tc_kernel_out || !nt_out)
        return set_error(RSATB_INVALID_ARGUMENT, "need at least one size and the outputs");
    if (problems_per_size < 1 || problems_per_size > 4096)
        return set_error(RSATB_INVALID_ARGUMENT, "problems_per_size outside [1, 4096]");
    for (int s = 0; s < n_sizes; ++s)
        if (sizes[s] < 1 || sizes[s] > 1024)
            return set_error(RSATB_INVALID_ARGUMENT, "size %d outside [1, 1024]", sizes[s]);

    std::vector<double> ms(size_t(n_sizes) * 8, -1.0);
    for (int si = 0; si < n_sizes; ++si) {
        const int n = sizes[si], np = (n + 31) / 32 * 32, count = problems_per_size;
        const int k = std::min(n, 16);
        std::vector<int64_t> in_off(count), out_off(count);
        std::vector<int32_t> nv(count, n), cs(count, 0), kc(count, k);
        for (int p = 0; p < count; ++p) {
            in_off[p] = int64_t(p) * n * n;
            out_off[p] = int64_t(p) * n * k;
        }
        double* M = nullptr;
        double* out = nullptr;
        RSATB_CUDA_TRY(cudaMalloc(&M, sizeof(double) * size_t(count) * n * n));
        cudaError_t ae = cudaMalloc(&out, sizeof(double) * size_t(count) * n * k);
        if (ae != cudaSuccess) {
            cudaFree(M);
            RSATB_CUDA_TRY(ae);
        }
        struct Free {
            double *a, *b;
            ~Free() {
                cudaFree(a);
                cudaFree(b);
            }
        } guard{M, out};
        spd_sample_kernel<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>(M, n, count,
                                                                     0x5EEDull + uint64_t(si));
        RSATB_LAUNCH_CHECK(ctx);
        std::vector<int32_t> status(count);
        for (int kk = 0; kk < 2; ++kk) {
            const bool ws = kk == 0;
            for (int idx = 0; idx < 4; ++idx) {
                int32_t nt = candidate_nt(np, ws, idx);
                if (!nt) continue;
                int32_t npad = np;
                rsatb_isqrt_options o{};
                o.precision = precision;
                o.max_iter = 6;        // a fixed-length solve: every candidate does the same work
                o.max_fp64_iter = 1;
                o.tol = 1e-300;
                o.tc_kernel = ws ? 1 : 2;
                o.n_tiles = 1;
                o.tile_n_pad = &npad;
                o.tile_nt = &nt;
                double best = 1e30;
                for (int rep = 0; rep < 3; ++rep) {
                    rsatb_isqrt_stats st{};
                    RSATB_TRY(rsatb_isqrt_columns_batched(ctx, count, nv.data(), cs.data(),
                                                          kc.data(), in_off.data(), M,
                                                          out_off.data(), out, &o, status.data(),
                                                          &st));
                    if (rep > 0) best = std::min(best, st.low_ms + st.fp64_ms);
                }
                ms[size_t(si) * 8 + kk * 4 + idx] = best;
            }
        }
    }
    // The kernel family, then its best tile per size.  The built-in family
    // (the warp-specialised kernel) stays unless the other one is faster by
    // more than 15 % on the samples: a few problems per size hide what the
    // warp specialisation buys on full chunks (the epilogue of one tile under
    // the main loop of the next), and a noisy pick of the single-role kernel
    // cost a quarter of the throughput of the 100,000-problem batch.
    double total[2] = {0.0, 0.0};
    for (int si = 0; si < n_sizes; ++si)
        for (int kk = 0; kk < 2; ++kk) {
            double b = 1e30;
            for (int idx = 0; idx < 4; ++idx) {
                const double t = ms[size_t(si) * 8 + kk * 4 + idx];
                if (t >= 0) b = std::min(b, t);
            }
            total[kk] += b;
        }
    const int builtin = default_tc_ws() ? 0 : 1, other = 1 - builtin;
    const int kk = total[other] < 0.85 * total[builtin] ? other : builtin;
    *tc_kernel_out = kk + 1;
    for (int si = 0; si < n_sizes; ++si) {
        const int np = (sizes[si] + 31) / 32 * 32;
        double b = 1e30;
        int best_nt = 0;
        for (int idx = 0; idx < 4; ++idx) {
            const double t = ms[size_t(si) * 8 + kk * 4 + idx];
            if (t >= 0 && t < b) {
                b = t;
                best_nt = candidate_nt(np, kk == 0, idx);
            }
        }
        nt_out[si] = best_nt;
    }
    if (ms_out) std::copy(ms.begin(), ms.end(), ms_out);
    return RSATB_SUCCESS;
}
