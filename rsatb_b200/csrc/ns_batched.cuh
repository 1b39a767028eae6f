// Shared definitions of the batched dense Newton-Schulz inverse square root
// (isqrt_batched.cu drives it; ns_tc_gemm.cu holds the tcgen05 GEMM).
//
// Every problem of a chunk owns one n_pad x n_pad block (row-major, n_pad a
// multiple of 32, zero outside the valid n x n corner) at the same element
// offset `off` of every workspace array.  Problems of equal n_pad are
// contiguous (a "bucket"), so one 3-D tensor map (n_pad, n_pad, count)
// addresses a whole bucket for TMA.
#pragma once

#include "common.cuh"

#include <cuda.h>

namespace rsatb_b200 {
namespace ns {

struct Prob {
    int n;        // valid size
    int n_pad;    // padded size, multiple of 32
    int64_t off;  // element offset of the problem's block in every workspace array
};

// Per-problem iteration state (rsatb/calc/isqrtm.hpp:615-660 loop variables).
struct State {
    double norm;      // last ||X - I||_F
    double norm_pre;  // previous one (0 before the first step, as the reference)
    int count;        // updates done in the current phase
    int active;       // still iterating
    int retire;       // stopped at the control step just run
    int status;       // rsatb_status
    int cap;          // iteration cap of the current phase
    int restart;      // FP64 phase restarts from Z0 (the tensor-core phase failed)
    int lift;         // next P uses the lift polynomial (tensor-core phase, ||X - I||_F large)
};

// P = a I + b X + c X X^T.  The reference's polynomial (15/8, -5/4, 3/8),
// rsatb/calc/isqrtm.hpp:646-667, maps an eigenvalue x of X to
// x p(x)^2 = 1 + (5/8) e^3 at x = 1 + e (cubic) and lifts a small x by
// p(0)^2 = 3.52 per step.  The lift polynomial (5/2, -5/2, 1) is the member
// of the family p(1) = 1, p'(1) = -1/2 (x = 1 a fixed point with quadratic
// convergence, 1 + (5/4) e^2) with p(0)^2 = 6.25: it maps [0, 9/8] into
// itself (its maximum, 9/8, at x = 1/2), so from the start, where the scale
// puts every eigenvalue in (0, 1], it lifts the small ones in
// log(1/x) / log(6.25) steps instead of log(1/x) / log(3.52) without
// leaving [0, 9/8]; the cubic polynomial finishes from there.
struct PolyCoef {
    float a, b, c;
};
__host__ __device__ inline PolyCoef poly_coef(int lift) {
    return lift ? PolyCoef{2.5f, -2.5f, 1.0f} : PolyCoef{1.875f, -1.25f, 0.375f};
}

enum EpiMode { EPI_STORE = 0, EPI_RESID = 1, EPI_POLY = 2 };

// Tensor-core tile: rows m0..m0+127 and columns n0..n0+nt-1 of problem p,
// which is entry z of bucket `bucket`.
struct TcItem {
    int p, bucket, z, m0, n0, nt;
};

constexpr int kMaxBuckets = 16;

// TMA maps of one GEMM launch, per bucket: A operand (box 32 x 128) and B
// operand (box 32 x nt), each as the TF32 "hi" array and the residual "lo".
struct TcMaps {
    CUtensorMap a_hi[kMaxBuckets];
    CUtensorMap a_lo[kMaxBuckets];
    CUtensorMap b_hi[kMaxBuckets];
    CUtensorMap b_lo[kMaxBuckets];
};

struct TcArgs {
    const Prob* probs;
    const TcItem* items;
    int n_items;
    const State* state;      // state[p].active gates the tile
    float* c_hi;             // C = A B^T: TF32-rounded value
    float* c_lo;             // and the residual value - c_hi (exact)
    double* c64;             // optional FP64 copy of C (c_hi + c_lo), nullptr: none
    const float* xe_hi;      // EPI_POLY: X (hi + lo) for P = a I + b X + c X X^T (poly_coef)
    const float* xe_lo;
    double* res2;            // EPI_RESID: per-problem sum of (C - I)^2 over the valid corner
    float* ct_hi;            // optional transposed store of C (hi, lo), nullptr: none
    float* ct_lo;
    int sym;                 // 1: only (row, col >= row) is stored, each also at (col, row):
                             // C leaves exactly symmetric (the items cover the upper
                             // triangle of tiles only)
    int mode;
    int split;               // 1: hi*hi + hi*lo + lo*hi; 0: hi*hi
    unsigned* error;         // set non-zero when a bounded wait gave up
    const int* live;         // optional: 0 when no problem of the chunk is still iterating
                             // (the launch returns at once), nullptr: always run
};

// One batched C = A B^T on the tensor cores for the items of up to
// kMaxBuckets buckets (ns_tc_gemm.cu).  Maps describe A and B per bucket.
// ws: the warp-specialised kernel (N tile <= 128), else the single-role one.
int launch_tc_gemm(rsatb_context* ctx, const TcMaps& maps, const TcArgs& args, bool ws);
// Sets the kernel's shared-memory opt-in and resolves the tensor-map
// encoder; called on the current device before any capture.
int prepare_tc_gemm();
// The built-in kernel choice (warp-specialised unless RSATB_NS_TC=simple)
// and the widest N tile each kernel takes (128 or 256).
bool default_tc_ws();
inline int tc_max_nt(bool ws) { return ws ? 128 : 256; }

// cuTensorMapEncodeTiled of a bucket: fp32 array `base` (element offset
// already applied), dims (n_pad, n_pad, count), box (32, box_rows, 1),
// 128-byte swizzle, out-of-bounds rows zero-filled.
int encode_bucket_map(CUtensorMap* map, const float* base, int n_pad, int count, int box_rows);

}  // namespace ns
}  // namespace rsatb_b200
