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
};

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
    const float* xe_hi;      // EPI_POLY: X (hi + lo) for P = 1.875 I - 1.25 X + 0.375 X X^T
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
