// FFT-Chebyshev Kubo-Greenwood transport on the device: the
// dc_spectrum_fftcheb / accumulate_fftcheb_block path of
// rsatb/calc/fftcheb_transport.hpp:270-660, Greenwood and Bastin formulations.
//
// Per sample block (all R samples at once) and per section of rows:
//   left chain   l_m = T_m(Op~) psi,          stored as J_a l_m for a = x, y, z
//   right chains r_m^a = T_m(Op~) J_a psi,    stored as they are
// with J_a = -(1 / 2 hw) V_a (current, rsatb/calc/ac.hpp:35-60, through
// Chebyshev::apply_dual, cheby.hpp:249-291), then per row, axis and sample
// the DCT-III of (g_m / pi) x_m (fft.hpp:125-154) for both chains and the
// contraction K_k += sum conj(L3_k) R3_k / max(1e-14, 1 - eps_k^2)
// (fftcheb_transport.hpp:481-495).
//
// B200 layout (the reference's per-row FFTW layout is not kept):
// * the three right chains are one N x 3R panel ([row][axis][sample]), so a
//   moment is one wide fused step for them and one narrow one for l;
// * the stores are moment-major, S[m][axis][row][sample], so every moment's
//   rows land with coalesced writes;
// * the DCT-III of a chunk of rows is a strided batched inverse 2M-point
//   FFT (cuFFT, sequences interleaved: stride = batch) of the half-grid
//   phased even extension, built and read back with coalesced accesses;
// * the contraction gives each energy k to one CTA per chunk: no atomics,
//   the same summation order on every run;
// * at M = 2048 (Greenwood) the row stage is one hand-written kernel after a
//   coalesced gather: extension, 4096-point transform and contraction
//   without the FP64 extension buffer's round trips (greenwood_fused_kernel).
#include "cheb_kernels.cuh"

#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <type_traits>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a);
void kpm_kernel_weights(int kernel, int n, double* g);

namespace {

#define RSATB_CUFFT_TRY(call)                                                              \
    do {                                                                                   \
        cufftResult r_ = (call);                                                           \
        if (r_ != CUFFT_SUCCESS)                                                           \
            return set_error(RSATB_CUDA_ERROR, "%s failed (cufftResult %d)", #call, int(r_)); \
    } while (0)

// Right-chain panel from the three J_a psi buffers: P[row][a][s] = J[a][row][s].
template <typename T>
__global__ void pack_axes_kernel(int64_t n_rows, int R, const T* j0, const T* j1, const T* j2,
                                 T* panel) {
    const int64_t total = n_rows * 3 * R;  // complex entries
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int s = int(e % R);
        const int a = int((e / R) % 3);
        const int64_t row = e / (3 * int64_t(R));
        const T* src = a == 0 ? j0 : (a == 1 ? j1 : j2);
        panel[2 * e] = src[2 * (row * R + s)];
        panel[2 * e + 1] = src[2 * (row * R + s) + 1];
    }
}

// Rows [row0, row0 + rows) of the right panel into store slot m:
// S[m][a][row][s] (complex entries), slot size 3 * rows * R.
template <typename T>
__global__ void store_right_kernel(int64_t row0, int64_t rows, int R, const T* panel, T* slot) {
    const int64_t total = rows * 3 * R;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        // e indexes the destination: a-major
        const int s = int(e % R);
        const int64_t row = (e / R) % rows;
        const int a = int(e / (rows * R));
        const int64_t src = ((row0 + row) * 3 + a) * R + s;
        slot[2 * e] = panel[2 * src];
        slot[2 * e + 1] = panel[2 * src + 1];
    }
}

// The same copy in 16-byte units: the R samples of one (row, axis) are one
// contiguous run in both layouts, of 2 R sizeof(T) / 16 units (R even for
// FP32; every run, slot and panel then starts on a 16-byte boundary).
template <typename T>
__global__ void store_right_vec_kernel(int64_t row0, int64_t rows, int R, const T* panel,
                                       T* slot) {
    const int upr = int(2 * R * sizeof(T) / 16);  // units per run
    const int64_t total = rows * 3 * upr;
    const float4* src = reinterpret_cast<const float4*>(panel);
    float4* dst = reinterpret_cast<float4*>(slot);
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int u = int(e % upr);
        const int64_t run = e / upr;  // destination run a * rows + row
        const int64_t row = run % rows;
        const int a = int(run / rows);
        dst[e] = src[((row0 + row) * 3 + a) * upr + u];
    }
}

// Even extension with the half-grid phase of fft.hpp:125-154 for a chunk of
// sequences: sequence q (0 <= q < nq, q = (a * chunk_rows + row) * R + s,
// rows offset row_off inside the section) of store S (slot stride
// slot_elems complex entries, section rows sec_rows) weighted by w_m:
//   E[0][q] = w_0 x_0,   E[m][q] = w_m x_m e^{i pi m / 2M},
//   E[2M - m][q] = w_m x_m e^{-i pi m / 2M}  (1 <= m < M),   E[M][q] = 0.
template <typename T>
__global__ void extend_kernel(int M, int64_t nq, int chunk_rows, int R, int64_t sec_rows,
                              int64_t row_off, int64_t slot_elems, const T* S, const double* w,
                              double2* E) {
    const int m = blockIdx.y;
    const double th = M_PI * double(m) / (2.0 * double(M));
    const double c = cos(th), sn = sin(th);
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < nq;
         q += int64_t(gridDim.x) * blockDim.x) {
        const int s = int(q % R);
        const int64_t row = (q / R) % chunk_rows;
        const int a = int(q / (int64_t(chunk_rows) * R));
        const int64_t src = int64_t(m) * slot_elems + (a * sec_rows + row_off + row) * R + s;
        const double xr = w[m] * double(S[2 * src]), xi = w[m] * double(S[2 * src + 1]);
        if (m == 0) {
            E[q] = make_double2(xr, xi);
            E[int64_t(M) * nq + q] = make_double2(0.0, 0.0);
        } else {
            E[int64_t(m) * nq + q] = make_double2(xr * c - xi * sn, xr * sn + xi * c);
            E[int64_t(2 * M - m) * nq + q] = make_double2(xr * c + xi * sn, -xr * sn + xi * c);
        }
    }
}

// Bastin phi1 / phi2 inputs (fftcheb_transport.hpp:453-461, fft.hpp:156-174):
// the weighted moments w[m] S_m (complex w) in the first M points of a
// 2M-point sequence, zeros in the last M.  Layout as extend_kernel.
template <typename T>
__global__ void pad_kernel(int M, int64_t nq, int chunk_rows, int R, int64_t sec_rows,
                           int64_t row_off, int64_t slot_elems, const T* S, const double2* w,
                           double2* E) {
    const int m = blockIdx.y;
    const double2 wm = w[m];
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < nq;
         q += int64_t(gridDim.x) * blockDim.x) {
        const int s = int(q % R);
        const int64_t row = (q / R) % chunk_rows;
        const int a = int(q / (int64_t(chunk_rows) * R));
        const int64_t src = int64_t(m) * slot_elems + (a * sec_rows + row_off + row) * R + s;
        const double xr = double(S[2 * src]), xi = double(S[2 * src + 1]);
        E[int64_t(m) * nq + q] = make_double2(wm.x * xr - wm.y * xi, wm.x * xi + wm.y * xr);
        E[int64_t(M + m) * nq + q] = make_double2(0.0, 0.0);
    }
}

// Bastin kernel accumulation (fftcheb_transport.hpp:496-519): for energy k
// (one CTA) and every component (a, b), a <= b,
//   K[k][ab] += sum over rows, samples of
//     eps_k (conj(L3_a) R1_b + conj(L1_a) R3_b)
//     + i sqrt(1 - eps_k^2) (conj(L2_a) R3_b - conj(L3_a) R2_b),
// summed per thread, then in a fixed tree order (deterministic).
__global__ void __launch_bounds__(256) bastin_contract_kernel(int M, int64_t nq, int64_t per_axis,
                                                              const double2* L3, const double2* R3,
                                                              const double2* L1, const double2* R1,
                                                              const double2* L2, const double2* R2,
                                                              double* K) {
    const int k = blockIdx.x;
    const double th = M_PI * (double(k) + 0.5) / double(M);
    const double eps = cos(th), root = sin(th);
    __shared__ double red[12][256];
    double acc[6][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
    const int64_t o = int64_t(k) * nq;
    // conj(x) y, accumulated into (re, im)
    auto cmac = [](double (&d)[2], double2 x, double2 y, double f_re, double f_im) {
        const double re = x.x * y.x + x.y * y.y, im = x.x * y.y - x.y * y.x;
        d[0] += f_re * re - f_im * im;
        d[1] += f_re * im + f_im * re;
    };
    for (int64_t q = threadIdx.x; q < per_axis; q += blockDim.x) {
        int comp = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double2 l3 = L3[o + a * per_axis + q], l1 = L1[o + a * per_axis + q],
                          l2 = L2[o + a * per_axis + q];
#pragma unroll
            for (int b = a; b < 3; ++b, ++comp) {
                const double2 r3 = R3[o + b * per_axis + q], r1 = R1[o + b * per_axis + q],
                              r2 = R2[o + b * per_axis + q];
                cmac(acc[comp], l3, r1, eps, 0.0);
                cmac(acc[comp], l1, r3, eps, 0.0);
                cmac(acc[comp], l2, r3, 0.0, root);
                cmac(acc[comp], l3, r2, 0.0, -root);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        red[2 * c][threadIdx.x] = acc[c][0];
        red[2 * c + 1][threadIdx.x] = acc[c][1];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 12; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 12) K[int64_t(k) * 12 + threadIdx.x] += red[threadIdx.x][0];
}

// K[k][a] += sum over the chunk's (row, s) of conj(L3[k][q]) R3[k][q] /
// max(1e-14, 1 - eps_k^2): one CTA per energy k, fixed order.
__global__ void __launch_bounds__(256) greenwood_contract_kernel(int M, int64_t nq,
                                                                 int64_t per_axis,
                                                                 const double2* L3,
                                                                 const double2* R3,
                                                                 double* K) {
    const int k = blockIdx.x;
    const double eps = cos(M_PI * (double(k) + 0.5) / double(M));
    const double wden = 1.0 - eps * eps;
    const double inv = 1.0 / (wden > 1e-14 ? wden : 1e-14);
    __shared__ double red[3][2][256];
    double acc[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    const double2* l = L3 + int64_t(k) * nq;
    const double2* r = R3 + int64_t(k) * nq;
    for (int a = 0; a < 3; ++a)
        for (int64_t q = threadIdx.x; q < per_axis; q += blockDim.x) {
            const double2 x = l[a * per_axis + q], y = r[a * per_axis + q];
            acc[a][0] += x.x * y.x + x.y * y.y;
            acc[a][1] += x.x * y.y - x.y * y.x;
        }
    for (int a = 0; a < 3; ++a) {
        red[a][0][threadIdx.x] = acc[a][0];
        red[a][1][threadIdx.x] = acc[a][1];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int a = 0; a < 3; ++a) {
                red[a][0][threadIdx.x] += red[a][0][threadIdx.x + w];
                red[a][1][threadIdx.x] += red[a][1][threadIdx.x + w];
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int a = 0; a < 3; ++a) {
            // components xx, yy, zz of the 6-component tensor (xx xy xz yy yz zz)
            const int comp = a == 0 ? 0 : (a == 1 ? 3 : 5);
            K[2 * (int64_t(k) * 6 + comp)] += red[a][0][0] * inv;
            K[2 * (int64_t(k) * 6 + comp) + 1] += red[a][1][0] * inv;
        }
}

// ---------------------------------------------------------------------------
// Fused Greenwood row stage for M = 2048 (a 4096-point transform): the even
// extension, the DCT-III (the inverse 2M-point DFT of extend_kernel's
// sequence, outputs k < M) and the contraction in one kernel, so no
// extended sequence or transform output goes through HBM.  The transform
// runs in FP64 for FP64 vectors and in FP32 for FP32 vectors; the products
// conj(L3) R3 and their sums are FP64 in both.
//
// One CTA of 256 threads transforms one sequence at a time as 16 x 16 x 16
// (n = n0 + 16 n1 + 256 n2, k = k0 + 16 k1 + 256 k2, w = e^{2 pi i / 4096}):
//   pass A  thread (n0, n1): 16-point DFT over n2 -> k0, times w^{(n0 + 16 n1) k0}
//   pass B  thread (n0, k0): 16-point DFT over n1 -> k1, times w^{16 n0 k1}
//   pass C  thread (k0, k1): 16-point DFT over n0 -> k2; k < 2048 is k2 < 8
// with the values between passes exchanged through shared memory (planes of
// 257 entries, so the 16-byte accesses of a quarter warp fall on distinct
// banks).  Pass A builds the extension as it loads: E_n = ph_n x_n (n < M),
// 0 (n = M), conj(ph_{2M-n}) x_{2M-n} (n > M), ph_m = w_m e^{i pi m / 2M}.
// Each thread keeps the left sequence's 8 outputs, transforms the right
// sequence and accumulates conj(L3_k) R3_k for its 8 energies in FP64 over
// the CTA's sequences (a fixed grid-stride order); fused_reduce_kernel sums
// the CTAs in a fixed order, so results do not depend on timing.
//
// The store is moment-major (each moment's rows written coalesced by the
// recurrence), so one sequence is 2048 values 8 or 16 bytes apiece at a
// stride of the slot size; gather_sequences_kernel first turns a chunk of
// consecutive sequences into sequence-major rows with a tiled transpose
// (both sides coalesced), from which pass A reads 256 contiguous values per
// warp instruction.
constexpr int kFusedM = 2048;
constexpr int kFusedThreads = 256;
constexpr int kXchPlane = 257;
// Shared memory of the fused kernel: exchange planes, w^j (j < 1024), ph.
template <typename C>
constexpr size_t fused_smem() {
    return size_t(16 * kXchPlane + 1024 + kFusedM) * sizeof(C);
}

// Complex arithmetic on float2 (FP32 transform) and double2 (FP64 transform).
template <typename C> struct Cx;
template <> struct Cx<float2> {
    using S = float;
    __device__ static float2 make(float x, float y) { return make_float2(x, y); }
};
template <> struct Cx<double2> {
    using S = double;
    __device__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <typename C>
__device__ __forceinline__ C c_add(C a, C b) {
    return Cx<C>::make(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C c_sub(C a, C b) {
    return Cx<C>::make(a.x - b.x, a.y - b.y);
}
template <typename C>
__device__ __forceinline__ C c_mul(C a, C b) {
    return Cx<C>::make(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C c_mul_i(C a) {
    return Cx<C>::make(-a.y, a.x);
}

// out[k] = sum_j in[j] i^{jk}, k = 0..3, in place.
template <typename C>
__device__ __forceinline__ void dft4_inv(C& a0, C& a1, C& a2, C& a3) {
    const C s02 = c_add(a0, a2), d02 = c_sub(a0, a2);
    const C s13 = c_add(a1, a3), d13 = c_mul_i(c_sub(a1, a3));
    a0 = c_add(s02, s13);
    a2 = c_sub(s02, s13);
    a1 = c_add(d02, d13);
    a3 = c_sub(d02, d13);
}

// 16-point DFT with the + sign, in place, as 4 x 4: j = j0 + 4 j1,
// k = c + 4 r.  Output k sits at v[4 (k % 4) + k / 4] (dft16_at).
template <typename C>
__device__ __forceinline__ void dft16_inv(C (&v)[16]) {
    using S = typename Cx<C>::S;
    constexpr S c8 = S(0.92387953251128674);  // cos(pi / 8)
    constexpr S s8 = S(0.38268343236508978);  // sin(pi / 8)
    constexpr S r2 = S(0.70710678118654752);  // cos(pi / 4)
#pragma unroll
    for (int j0 = 0; j0 < 4; ++j0) dft4_inv(v[j0], v[j0 + 4], v[j0 + 8], v[j0 + 12]);
    // v[j0 + 4 c] *= e^{2 pi i j0 c / 16}
    v[1 + 4] = c_mul(v[1 + 4], Cx<C>::make(c8, s8));     // 1
    v[2 + 4] = c_mul(v[2 + 4], Cx<C>::make(r2, r2));     // 2
    v[3 + 4] = c_mul(v[3 + 4], Cx<C>::make(s8, c8));     // 3
    v[1 + 8] = c_mul(v[1 + 8], Cx<C>::make(r2, r2));     // 2
    v[2 + 8] = c_mul_i(v[2 + 8]);                        // 4
    v[3 + 8] = c_mul(v[3 + 8], Cx<C>::make(-r2, r2));    // 6
    v[1 + 12] = c_mul(v[1 + 12], Cx<C>::make(s8, c8));   // 3
    v[2 + 12] = c_mul(v[2 + 12], Cx<C>::make(-r2, r2));  // 6
    v[3 + 12] = c_mul(v[3 + 12], Cx<C>::make(-c8, -s8)); // 9
#pragma unroll
    for (int c = 0; c < 4; ++c) dft4_inv(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
}
__device__ __forceinline__ int dft16_at(int k) { return 4 * (k & 3) + (k >> 2); }

// w^n = e^{2 pi i n / 4096} from the quarter table q[j] = w^j, j < 1024.
template <typename C>
__device__ __forceinline__ C twiddle4096(const C* q, int n) {
    const C b = q[n & 1023];
    switch ((n >> 10) & 3) {
        case 0: return b;
        case 1: return Cx<C>::make(-b.y, b.x);
        case 2: return Cx<C>::make(-b.x, -b.y);
        default: return Cx<C>::make(b.y, -b.x);
    }
}

// The powers b^k, k = 0..15, of a twiddle b as b4^(k / 4) b^(k % 4), from b
// and b4 = b^4 (two reads of the quarter table, whose strided lanes would
// otherwise conflict on the shared-memory banks sixteen at a time): at most
// four roundings more than a table entry.
template <typename C>
struct Pow16 {
    C lo[4], hi[4];
    __device__ __forceinline__ Pow16(C b, C b4) {
        lo[0] = hi[0] = Cx<C>::make(1, 0);
        lo[1] = b;
        lo[2] = c_mul(b, b);
        lo[3] = c_mul(lo[2], b);
        hi[1] = b4;
        hi[2] = c_mul(b4, b4);
        hi[3] = c_mul(hi[2], b4);
    }
    __device__ __forceinline__ C operator()(int k) const {
        if (k < 4) return lo[k];
        if ((k & 3) == 0) return hi[k >> 2];
        return c_mul(hi[k >> 2], lo[k & 3]);
    }
};

// Element e of a store as the transform's complex type.
template <typename C>
__device__ __forceinline__ C load_c(const float* S, int64_t e) {
    const float2 f = __ldg(reinterpret_cast<const float2*>(S) + e);
    return Cx<C>::make(typename Cx<C>::S(f.x), typename Cx<C>::S(f.y));
}
template <typename C>
__device__ __forceinline__ C load_c(const double* S, int64_t e) {
    const double2 f = __ldg(reinterpret_cast<const double2*>(S) + e);
    return Cx<C>::make(typename Cx<C>::S(f.x), typename Cx<C>::S(f.y));
}

// The 8 outputs k0 + 16 k1 + 256 k2 (k2 < 8) of thread (k0, k1) for the
// sequence whose element m is S[m + base] (complex index; sequence-major).
template <typename C, typename T>
__device__ __forceinline__ void fused_transform(const T* S, int64_t base, const C* qtw,
                                                const C* ph, C* xch, C (&out)[8]) {
    const int t = threadIdx.x;
    C v[16];
    // pass A: thread (n0, n1) = (t % 16, t / 16) holds E_{t + 256 n2}
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int n = t + 256 * j;
        if (j < 8) {
            v[j] = c_mul(ph[n], load_c<C>(S, base + n));
        } else if (n == kFusedM) {
            v[j] = Cx<C>::make(0, 0);
        } else {
            const int m = 2 * kFusedM - n;
            const C p = ph[m];
            v[j] = c_mul(Cx<C>::make(p.x, -p.y), load_c<C>(S, base + m));
        }
    }
    dft16_inv(v);
    {
        const int n0 = t & 15, n1 = t >> 4;
        const Pow16<C> tw(twiddle4096(qtw, t), twiddle4096(qtw, 4 * t));  // w^{t k0}
#pragma unroll
        for (int k0 = 0; k0 < 16; ++k0)
            xch[n0 * kXchPlane + k0 * 16 + n1] = c_mul(v[dft16_at(k0)], tw(k0));
    }
    __syncthreads();
    // pass B: thread (n0, k0) = (t % 16, t / 16)
    {
        const int n0 = t & 15, k0 = t >> 4;
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) v[n1] = xch[n0 * kXchPlane + k0 * 16 + n1];
        dft16_inv(v);
        const Pow16<C> tw(twiddle4096(qtw, 16 * n0), twiddle4096(qtw, 64 * n0));  // w^{16 n0 k1}
        __syncthreads();
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1)
            xch[k0 * kXchPlane + k1 * 16 + n0] = c_mul(v[dft16_at(k1)], tw(k1));
    }
    __syncthreads();
    // pass C: thread (k0, k1) = (t % 16, t / 16)
    {
        const int k0 = t & 15, k1 = t >> 4;
#pragma unroll
        for (int n0 = 0; n0 < 16; ++n0) v[n0] = xch[k0 * kXchPlane + k1 * 16 + n0];
        dft16_inv(v);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) out[k2] = v[dft16_at(k2)];
    }
    __syncthreads();  // xch is rewritten by the next transform
}

// The tables of the transform: tab[j] = w^j (j < 1024), tab[1024 + m] = ph_m.
__global__ void fused_tables_kernel(const double* w, double2* tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s, c;
    if (i < 1024) {
        sincospi(double(i) / 2048.0, &s, &c);  // w^j = e^{2 pi i j / 4096}
        tab[i] = make_double2(c, s);
    } else if (i < 1024 + kFusedM) {
        const int m = i - 1024;
        sincospi(double(m) / (2.0 * kFusedM), &s, &c);  // e^{i pi m / 2M}
        tab[i] = make_double2(w[m] * c, w[m] * s);
    }
}

// Tq[side][i][m] = S_side[m * slot + q0 + i] for i < nqc (complex entries):
// 32 x 32 tiles through shared memory, blockIdx.z the side (left, right).
template <typename T>
__global__ void __launch_bounds__(256) gather_sequences_kernel(int64_t q0, int64_t nqc,
                                                               int64_t slot, const T* SL,
                                                               const T* SR, T* Tq) {
    using C = typename std::conditional<std::is_same<T, float>::value, float2, double2>::type;
    __shared__ C tile[32][33];
    const C* S = reinterpret_cast<const C*>(blockIdx.z ? SR : SL);
    C* out = reinterpret_cast<C*>(Tq) + int64_t(blockIdx.z) * nqc * kFusedM;
    const int64_t i0 = int64_t(blockIdx.x) * 32;
    const int m0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int m = m0 + ty + 8 * r;
        if (i0 + tx < nqc) tile[ty + 8 * r][tx] = S[int64_t(m) * slot + q0 + i0 + tx];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int64_t i = i0 + ty + 8 * r;
        if (i < nqc) out[i * kFusedM + m0 + tx] = tile[tx][ty + 8 * r];
    }
}

// Gathered sequences i < nqc of one chunk (Tq, left then right), transform
// in the precision of C; partial[cta][k] += sum over the CTA's sequences of
// conj(L3_k) R3_k, the products and the sums in FP64.  Two CTAs per SM for
// the FP32 transform (half the registers and shared memory), one for FP64.
template <typename T, typename C>
__global__ void __launch_bounds__(kFusedThreads, sizeof(C) == 8 ? 2 : 1)
    greenwood_fused_kernel(int64_t nqc, const T* Tq, const double2* tab, double2* partial) {
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    C* xch = reinterpret_cast<C*>(fsm_raw);
    C* qtw = xch + 16 * kXchPlane;
    C* ph = qtw + 1024;
    for (int j = threadIdx.x; j < 1024 + kFusedM; j += blockDim.x)
        qtw[j] = Cx<C>::make(typename Cx<C>::S(tab[j].x), typename Cx<C>::S(tab[j].y));
    __syncthreads();
    double2 acc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = make_double2(0.0, 0.0);
    const int64_t right = nqc * kFusedM;
    for (int64_t i = blockIdx.x; i < nqc; i += gridDim.x) {
        C l3[8], r3[8];
        fused_transform(Tq, i * kFusedM, qtw, ph, xch, l3);
        fused_transform(Tq, right + i * kFusedM, qtw, ph, xch, r3);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const double lx = l3[j].x, ly = l3[j].y, rx = r3[j].x, ry = r3[j].y;
            acc[j].x += lx * rx + ly * ry;  // conj(L3) R3
            acc[j].y += lx * ry - ly * rx;
        }
    }
    double2* p = partial + int64_t(blockIdx.x) * kFusedM + threadIdx.x;
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) p[256 * k2] = make_double2(p[256 * k2].x + acc[k2].x,
                                                              p[256 * k2].y + acc[k2].y);
}

// K[k][comp] += sum over the n_cta partials (in CTA order) / max(1e-14, 1 - eps_k^2).
__global__ void fused_reduce_kernel(int n_cta, const double2* partial, int comp, double* K) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kFusedM) return;
    double re = 0.0, im = 0.0;
    for (int c = 0; c < n_cta; ++c) {
        const double2 p = partial[int64_t(c) * kFusedM + k];
        re += p.x;
        im += p.y;
    }
    const double eps = cos(M_PI * (double(k) + 0.5) / double(kFusedM));
    const double wden = 1.0 - eps * eps;
    const double inv = 1.0 / (wden > 1e-14 ? wden : 1e-14);
    K[2 * (int64_t(k) * 6 + comp)] += re * inv;
    K[2 * (int64_t(k) * 6 + comp) + 1] += im * inv;
}

// The fused row stage serves Greenwood at M = 2048 unless RSATB_FFTCHEB_FUSED=0.
bool fused_enabled() {
    const char* s = std::getenv("RSATB_FFTCHEB_FUSED");
    return !(s && s[0] == '0');
}

// RSATB_FFTCHEB_FP64=1: the FP64 transform for FP32 vectors too.
bool fused_fp64_forced() {
    const char* s = std::getenv("RSATB_FFTCHEB_FP64");
    return s && s[0] == '1';
}

// Owning device buffer released on scope exit.
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    int alloc(size_t bytes) {
        if (bytes == 0) bytes = 16;
        RSATB_CUDA_TRY(cudaMalloc(&p, bytes));
        return RSATB_SUCCESS;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct Plan {
    cufftHandle h = 0;
    bool made = false;
    ~Plan() {
        if (made) cufftDestroy(h);
    }
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

StepArgs plain_args(int W) {
    StepArgs a{};
    a.W = W;
    a.s_in = 1.0;
    a.s_out = 1.0;
    a.s2 = 1.0;
    a.dot_mode = DOT_NONE;
    return a;
}

// Matrix restricted to block rows [b0, b1): row_ptr keeps absolute block
// indices, so values, column indices and the input panel are unchanged and
// output row i of the launch is block row b0 + i.
rsatb_bsr_matrix row_view(const rsatb_bsr_matrix* A, int b0, int b1) {
    rsatb_bsr_matrix v = *A;
    v.row_ptr = A->row_ptr + b0;
    v.n_block_rows = b1 - b0;
    return v;
}

struct Ctx {
    rsatb_context* ctx;
    const rsatb_cheb_op* op;
    bool sandwich;
    int vdt;
};

// out = s2 * (Op in - c in) / hw + g_p * prev (Chebyshev::apply_form and the
// recurrence axpby), W real values per row; u, w: sandwich scratch.
int op_step(const Ctx& c, int W, const void* in, const void* prev, void* out, void* u, void* w,
            double s2, double g_p) {
    StepArgs last = plain_args(W);
    last.x = in;
    last.p = prev;
    last.y = out;
    last.c = c.op->center;
    last.s_out = 1.0 / c.op->half_width;
    last.s2 = s2;
    last.g_p = g_p;
    if (!c.sandwich) {
        last.in = in;
        return run_step(c.ctx, c.op->H, c.vdt, last);
    }
    StepArgs a = plain_args(W);
    a.in = in;
    a.y = u;
    RSATB_TRY(run_step(c.ctx, c.op->Z, c.vdt, a));
    a.in = u;
    a.y = w;
    RSATB_TRY(run_step(c.ctx, c.op->H, c.vdt, a));
    last.in = w;
    return run_step(c.ctx, c.op->ZH, c.vdt, last);
}

// J_a x = -(1 / 2 hw) * (dressed V_a) x on block rows [b0, b1), written
// compactly to out (rows b0.. of the result at out[0..]).  Sandwich: Z^H V Z.
int current_rows(const Ctx& c, const rsatb_bsr_matrix* V, int W, const void* x, void* out,
                 int b0, int b1, void* u, void* w) {
    const double scale = -1.0 / (2.0 * c.op->half_width);
    StepArgs a = plain_args(W);
    if (!c.sandwich) {
        const rsatb_bsr_matrix view = row_view(V, b0, b1);
        a.in = x;
        a.y = out;
        a.s_in = scale;
        return run_step(c.ctx, &view, c.vdt, a);
    }
    a.in = x;
    a.y = u;
    RSATB_TRY(run_step(c.ctx, c.op->Z, c.vdt, a));
    a.in = u;
    a.y = w;
    RSATB_TRY(run_step(c.ctx, V, c.vdt, a));
    const rsatb_bsr_matrix view = row_view(c.op->ZH, b0, b1);
    a.in = w;
    a.y = out;
    a.s_in = scale;
    return run_step(c.ctx, &view, c.vdt, a);
}

unsigned grid_for(int64_t n, int sm) {
    int64_t g = (n + 255) / 256;
    if (g > int64_t(sm) * 16) g = int64_t(sm) * 16;
    return unsigned(g < 1 ? 1 : g);
}

template <typename T>
int fftcheb_impl(const Ctx& c, const rsatb_bsr_matrix* const* V, const T* psi, int R, int M,
                 int formulation, double prefactor, int sections, size_t workspace, int kernel,
                 double* sigma_out, double* energy_out, rsatb_fftcheb_stats* stats) {
    const bool bastin = formulation == 1;
    const int n_tf = bastin ? 3 : 1;  // transforms per side and row: phi3 (+ phi1, phi2)
    rsatb_context* ctx = c.ctx;
    cudaStream_t st = ctx->stream;
    const int b = c.op->H->block_size;
    const int nb = c.op->H->n_block_rows;
    const int64_t N = int64_t(nb) * b;
    const int W1 = 2 * R, W3 = 6 * R;  // real values per row: left, right panel
    const size_t cplx = 2 * sizeof(T);

    // Store per block row: both chains, all moments, 3 axes x R samples.
    const size_t store_per_brow = 2 * size_t(M) * b * 3 * R * cplx;
    const size_t fixed = size_t(N) * cplx * (3 * R /*rinit*/ + 3 * 3 * R /*r*/ + 3 * R /*l*/ +
                                            3 * R /*J psi*/ + (c.sandwich ? 2 * 3 * R : 0));
    if (workspace == 0) {
        size_t free_b = 0, total_b = 0;
        RSATB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        workspace = free_b / 10 * 8;
    }
    if (workspace <= fixed + store_per_brow)
        return set_error(RSATB_OUT_OF_MEMORY,
                         "workspace of %zu bytes holds no section (needs %zu + %zu per block row)",
                         workspace, fixed, store_per_brow);
    // FFT chunk: rows whose 2 x (2M x 3 rows R) double2 extensions fit a
    // quarter of what remains after the fixed buffers.  The fused row stage
    // (Greenwood, M = 2048) needs only its gathered chunk of up to 8,192
    // sequence pairs, and the store takes the rest (larger sections: fewer
    // passes of the recurrence).
    const size_t avail = workspace - fixed;
    const bool fused = !bastin && M == kFusedM && fused_enabled();
    const size_t fused_chunk_bytes = 2 * size_t(8192) * size_t(M) * cplx;
    const size_t fft_budget =
        fused ? std::max(2 * size_t(M) * cplx, std::min(avail / 4, fused_chunk_bytes))
              : avail / 4;
    const size_t fft_per_row =
        size_t(n_tf) * 2 * 2 * size_t(M) * 3 * R * sizeof(double2) * 2;  // + cuFFT work
    int64_t chunk_rows = int64_t(fft_budget / fft_per_row);
    if (chunk_rows < 1) chunk_rows = 1;
    int64_t sec_brows = int64_t((avail - fft_budget) / store_per_brow);
    if (sec_brows < 1)
        return set_error(RSATB_OUT_OF_MEMORY, "workspace too small for one block row of stores");
    if (sections > 0) {
        const int64_t want = (nb + sections - 1) / sections;
        if (want < sec_brows) sec_brows = want;
    }
    if (sec_brows > nb) sec_brows = nb;
    const int n_sections = int((nb + sec_brows - 1) / sec_brows);
    sec_brows = (nb + n_sections - 1) / n_sections;  // balanced: the store is no larger than needed
    if (chunk_rows > sec_brows * b) chunk_rows = sec_brows * b;

    // Buffers.
    DevBuf bJ, bRinit, bR, bL, bU, bW, bS, bE, bK, bWts;
    RSATB_TRY(bJ.alloc(size_t(N) * 3 * R * cplx));
    RSATB_TRY(bRinit.alloc(size_t(N) * 3 * R * cplx));
    RSATB_TRY(bR.alloc(size_t(N) * 3 * 3 * R * cplx));
    RSATB_TRY(bL.alloc(size_t(N) * 3 * R * cplx));
    if (c.sandwich) {
        RSATB_TRY(bU.alloc(size_t(N) * 3 * R * cplx));
        RSATB_TRY(bW.alloc(size_t(N) * 3 * R * cplx));
    }
    const int64_t sec_rows_max = sec_brows * b;
    const int64_t slot = 3 * sec_rows_max * R;  // complex entries per moment slot
    RSATB_TRY(bS.alloc(2 * size_t(M) * slot * cplx));
    const int64_t nq_max = 3 * chunk_rows * R;
    const size_t e_bytes =
        fused ? fft_budget : size_t(n_tf) * 2 * 2 * size_t(M) * nq_max * sizeof(double2);
    RSATB_TRY(bE.alloc(e_bytes));
    RSATB_TRY(bK.alloc(size_t(M) * 12 * sizeof(double)));
    RSATB_TRY(bWts.alloc(size_t(M) * sizeof(double)));
    DevBuf bPw;
    if (bastin) RSATB_TRY(bPw.alloc(2 * size_t(M) * sizeof(double2)));
    T* J[3];
    for (int a = 0; a < 3; ++a) J[a] = bJ.as<T>() + size_t(a) * N * 2 * R;
    T* rinit = bRinit.as<T>();
    T* r[3];
    T* l[3];
    for (int i = 0; i < 3; ++i) {
        r[i] = bR.as<T>() + size_t(i) * N * 6 * R;
        l[i] = bL.as<T>() + size_t(i) * N * 2 * R;
    }
    T* SL = bS.as<T>();
    T* SR = SL + 2 * size_t(M) * slot;
    double2* EL = bE.as<double2>();
    double2* ER = fused ? nullptr : EL + 2 * size_t(M) * nq_max;
    // Bastin: phi1 and phi2 of both sides follow.
    double2* EL1 = bastin ? ER + 2 * size_t(M) * nq_max : nullptr;
    double2* ER1 = bastin ? EL1 + 2 * size_t(M) * nq_max : nullptr;
    double2* EL2 = bastin ? ER1 + 2 * size_t(M) * nq_max : nullptr;
    double2* ER2 = bastin ? EL2 + 2 * size_t(M) * nq_max : nullptr;
    double* K = bK.as<double>();

    std::vector<double> g(M), wts(M);
    kpm_kernel_weights(kernel, M, g.data());
    for (int m = 0; m < M; ++m) wts[m] = g[m] / M_PI;  // phi3_weight (fftcheb_transport.hpp)
    RSATB_CUDA_TRY(cudaMemcpyAsync(bWts.p, wts.data(), M * sizeof(double),
                                   cudaMemcpyHostToDevice, st));
    // Bastin phase weights (fftcheb_transport.hpp:302-310): phase_weight[m] =
    // 2 g_m / (pi (1 + [m == 0])) e^{i pi m / 2M}, phase_weight_m = m times it.
    std::vector<double2> pw;
    if (bastin) {
        pw.resize(2 * size_t(M));
        for (int m = 0; m < M; ++m) {
            const double coeff = 2.0 * g[m] / (M_PI * (1.0 + (m == 0 ? 1.0 : 0.0)));
            const double th = M_PI * double(m) / (2.0 * double(M));
            pw[m] = make_double2(coeff * std::cos(th), coeff * std::sin(th));
            pw[M + m] = make_double2(pw[m].x * double(m), pw[m].y * double(m));
        }
        RSATB_CUDA_TRY(cudaMemcpyAsync(bPw.p, pw.data(), pw.size() * sizeof(double2),
                                       cudaMemcpyHostToDevice, st));
    }
    RSATB_CUDA_TRY(cudaMemsetAsync(K, 0, size_t(M) * 12 * sizeof(double), st));

    // Fused row stage (Greenwood, M = 2048): one CTA per SM, partial sums
    // per CTA and energy; chunks of fused_qc sequences gathered into the
    // extension buffer (sequence-major, both sides).
    // FP32 vectors take the FP32 transform (FP64 products and sums) unless
    // RSATB_FFTCHEB_FP64=1; FP64 vectors the FP64 one.
    const bool fused32 = fused && std::is_same<T, float>::value && !fused_fp64_forced();
    const int fused_grid = ctx->sm_count * (fused32 ? 2 : 1);
    int64_t fused_qc = std::max<int64_t>(
        1, std::min<int64_t>(8192, int64_t(e_bytes / (2 * size_t(M) * cplx))));
    if (const char* cap = std::getenv("RSATB_FFTCHEB_CHUNK")) {  // smaller chunks (tests)
        const int64_t c = std::atoll(cap);
        if (c > 0 && c < fused_qc) fused_qc = c;
    }
    DevBuf bPart, bTab;
    if (fused) {
        RSATB_TRY(bPart.alloc(size_t(fused_grid) * kFusedM * sizeof(double2)));
        RSATB_TRY(bTab.alloc(size_t(1024 + kFusedM) * sizeof(double2)));
        fused_tables_kernel<<<(1024 + kFusedM) / 256, 256, 0, st>>>(bWts.as<double>(),
                                                                    bTab.as<double2>());
        RSATB_LAUNCH_CHECK(ctx);
        RSATB_CUDA_TRY(cudaFuncSetAttribute(greenwood_fused_kernel<T, double2>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(fused_smem<double2>())));
        if constexpr (std::is_same<T, float>::value)
            RSATB_CUDA_TRY(cudaFuncSetAttribute(greenwood_fused_kernel<T, float2>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                int(fused_smem<float2>())));
    }

    // cuFFT plans: full chunks and the last, shorter chunk of a section.
    Plan plans[2];
    int64_t plan_nq[2] = {0, 0};
    auto plan_for = [&](int64_t nq, cufftHandle* out) -> int {
        for (int i = 0; i < 2; ++i)
            if (plans[i].made && plan_nq[i] == nq) {
                *out = plans[i].h;
                return RSATB_SUCCESS;
            }
        int slot_i = plans[0].made ? 1 : 0;
        if (plans[slot_i].made) {
            cufftDestroy(plans[slot_i].h);
            plans[slot_i].made = false;
        }
        int n2 = 2 * M;
        int emb = 2 * M;
        RSATB_CUFFT_TRY(cufftPlanMany(&plans[slot_i].h, 1, &n2, &emb, int(nq), 1, &emb, int(nq), 1,
                                      CUFFT_Z2Z, int(nq)));
        plans[slot_i].made = true;
        plan_nq[slot_i] = nq;
        RSATB_CUFFT_TRY(cufftSetStream(plans[slot_i].h, st));
        *out = plans[slot_i].h;
        return RSATB_SUCCESS;
    };

    cudaEvent_t ev0, ev1;
    RSATB_CUDA_TRY(cudaEventCreate(&ev0));
    RSATB_CUDA_TRY(cudaEventCreate(&ev1));
    struct EvG {
        cudaEvent_t a, b;
        ~EvG() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evg{ev0, ev1};
    float rec_ms = 0.f, dct_ms = 0.f;

    // J_a psi and the right-chain start.
    for (int a = 0; a < 3; ++a)
        RSATB_TRY(current_rows(c, V[a], W1, psi, J[a], 0, nb, bU.p, bW.p));
    pack_axes_kernel<T><<<grid_for(N * 3 * R, ctx->sm_count), 256, 0, st>>>(N, R, J[0], J[1],
                                                                           J[2], rinit);
    RSATB_LAUNCH_CHECK(ctx);

    int64_t chunks = 0;
    for (int sec = 0; sec < n_sections; ++sec) {
        const int sb0 = int(sec * sec_brows);
        const int sb1 = int(std::min<int64_t>(nb, sb0 + sec_brows));
        const int64_t rows0 = int64_t(sb0) * b;
        const int64_t rows = int64_t(sb1 - sb0) * b;
        const int64_t sslot = 3 * rows * R;  // this section's slot size
        RSATB_CUDA_TRY(cudaEventRecord(ev0, st));
        RSATB_CUDA_TRY(cudaMemcpyAsync(r[0], rinit, size_t(N) * 3 * R * cplx,
                                       cudaMemcpyDeviceToDevice, st));
        const T* lp = psi;       // l_{m-1}
        const T* lc = nullptr;   // l_m
        int ri_prev = 0, ri_cur = -1;
        int li = 0;
        for (int m = 0; m < M; ++m) {
            const T* lm;  // l_m
            int rm;       // index of r_m
            if (m == 0) {
                lm = psi;
                rm = 0;
            } else if (m == 1) {
                T* lo = l[li];
                li = (li + 1) % 3;
                RSATB_TRY(op_step(c, W1, lp, nullptr, lo, bU.p, bW.p, 1.0, 0.0));
                RSATB_TRY(op_step(c, W3, r[ri_prev], nullptr, r[1], bU.p, bW.p, 1.0, 0.0));
                lc = lo;
                ri_cur = 1;
                lm = lc;
                rm = 1;
            } else {
                T* lo = l[li];
                li = (li + 1) % 3;
                const int rn = 3 - ri_prev - ri_cur;
                RSATB_TRY(op_step(c, W1, lc, lp, lo, bU.p, bW.p, 2.0, -1.0));
                RSATB_TRY(op_step(c, W3, r[ri_cur], r[ri_prev], r[rn], bU.p, bW.p, 2.0, -1.0));
                lp = lc;
                lc = lo;
                ri_prev = ri_cur;
                ri_cur = rn;
                lm = lc;
                rm = rn;
            }
            T* sl = SL + 2 * size_t(m) * sslot;
            for (int a = 0; a < 3; ++a)
                RSATB_TRY(current_rows(c, V[a], W1, lm, sl + 2 * size_t(a) * rows * R, sb0, sb1,
                                       bU.p, bW.p));
            if (sizeof(T) == 8 || R % 2 == 0)
                store_right_vec_kernel<T>
                    <<<grid_for(sslot * 2 * int64_t(sizeof(T)) / 16, ctx->sm_count), 256, 0, st>>>(
                        rows0, rows, R, r[rm], SR + 2 * size_t(m) * sslot);
            else
                store_right_kernel<T><<<grid_for(sslot, ctx->sm_count), 256, 0, st>>>(
                    rows0, rows, R, r[rm], SR + 2 * size_t(m) * sslot);
            RSATB_LAUNCH_CHECK(ctx);
        }
        RSATB_CUDA_TRY(cudaEventRecord(ev1, st));
        RSATB_CUDA_TRY(cudaEventSynchronize(ev1));
        float t = 0.f;
        cudaEventElapsedTime(&t, ev0, ev1);
        rec_ms += t;

        // Row stage: fused at M = 2048 (Greenwood), else in chunks of rows
        // through the extension, cuFFT and the contraction.
        RSATB_CUDA_TRY(cudaEventRecord(ev0, st));
        if (fused) {
            const int64_t per_axis = rows * R;
            T* Tq = reinterpret_cast<T*>(EL);
            for (int a = 0; a < 3; ++a) {
                RSATB_CUDA_TRY(cudaMemsetAsync(
                    bPart.p, 0, size_t(fused_grid) * kFusedM * sizeof(double2), st));
                for (int64_t i0 = 0; i0 < per_axis; i0 += fused_qc) {
                    const int64_t n = std::min<int64_t>(fused_qc, per_axis - i0);
                    const dim3 gg(unsigned((n + 31) / 32), kFusedM / 32, 2);
                    gather_sequences_kernel<T><<<gg, 256, 0, st>>>(int64_t(a) * per_axis + i0, n,
                                                                   sslot, SL, SR, Tq);
                    RSATB_LAUNCH_CHECK(ctx);
                    bool done = false;
                    if constexpr (std::is_same<T, float>::value) {
                        if (fused32) {
                            greenwood_fused_kernel<T, float2>
                                <<<fused_grid, kFusedThreads, fused_smem<float2>(), st>>>(
                                    n, Tq, bTab.as<double2>(), bPart.as<double2>());
                            done = true;
                        }
                    }
                    if (!done)
                        greenwood_fused_kernel<T, double2>
                            <<<fused_grid, kFusedThreads, fused_smem<double2>(), st>>>(
                                n, Tq, bTab.as<double2>(), bPart.as<double2>());
                    RSATB_LAUNCH_CHECK(ctx);
                    ++chunks;
                }
                fused_reduce_kernel<<<kFusedM / 256, 256, 0, st>>>(
                    fused_grid, bPart.as<double2>(), a == 0 ? 0 : (a == 1 ? 3 : 5), K);
                RSATB_LAUNCH_CHECK(ctx);
            }
        }
        for (int64_t c0 = 0; !fused && c0 < rows; c0 += chunk_rows) {
            const int64_t cr = std::min<int64_t>(chunk_rows, rows - c0);
            const int64_t nq = 3 * cr * R;
            cufftHandle plan;
            RSATB_TRY(plan_for(nq, &plan));
            dim3 grid(grid_for(nq, ctx->sm_count) > 64 ? 64 : grid_for(nq, ctx->sm_count), M);
            extend_kernel<T><<<grid, 256, 0, st>>>(M, nq, int(cr), R, rows, c0, sslot, SL,
                                                   bWts.as<double>(), EL);
            RSATB_LAUNCH_CHECK(ctx);
            extend_kernel<T><<<grid, 256, 0, st>>>(M, nq, int(cr), R, rows, c0, sslot, SR,
                                                   bWts.as<double>(), ER);
            RSATB_LAUNCH_CHECK(ctx);
            RSATB_CUFFT_TRY(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(EL),
                                         reinterpret_cast<cufftDoubleComplex*>(EL),
                                         CUFFT_INVERSE));
            RSATB_CUFFT_TRY(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(ER),
                                         reinterpret_cast<cufftDoubleComplex*>(ER),
                                         CUFFT_INVERSE));
            if (!bastin) {
                greenwood_contract_kernel<<<M, 256, 0, st>>>(M, nq, cr * R, EL, ER, K);
                RSATB_LAUNCH_CHECK(ctx);
            } else {
                const double2* w1 = bPw.as<double2>();
                const double2* w2 = w1 + M;
                double2* dst[4] = {EL1, ER1, EL2, ER2};
                const T* src[4] = {SL, SR, SL, SR};
                const double2* wt[4] = {w1, w1, w2, w2};
                for (int t = 0; t < 4; ++t) {
                    pad_kernel<T><<<grid, 256, 0, st>>>(M, nq, int(cr), R, rows, c0, sslot,
                                                        src[t], wt[t], dst[t]);
                    RSATB_LAUNCH_CHECK(ctx);
                    RSATB_CUFFT_TRY(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(dst[t]),
                                                 reinterpret_cast<cufftDoubleComplex*>(dst[t]),
                                                 CUFFT_INVERSE));
                }
                bastin_contract_kernel<<<M, 256, 0, st>>>(M, nq, cr * R, EL, ER, EL1, ER1, EL2,
                                                          ER2, K);
                RSATB_LAUNCH_CHECK(ctx);
            }
            ++chunks;
        }
        RSATB_CUDA_TRY(cudaEventRecord(ev1, st));
        RSATB_CUDA_TRY(cudaEventSynchronize(ev1));
        cudaEventElapsedTime(&t, ev0, ev1);
        dct_ms += t;
    }

    std::vector<double> Kh(size_t(M) * 12);
    RSATB_CUDA_TRY(cudaMemcpyAsync(Kh.data(), K, Kh.size() * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    RSATB_CUDA_TRY(cudaStreamSynchronize(st));
    RSATB_TRY(ctx_check_fault(ctx));
    // Sample average and the ascending energy grid of
    // fftcheb_transport.hpp:602-659: E_k = c + hw cos(pi (M - 1 - k + 1/2) / M).
    for (int k = 0; k < M; ++k) {
        const int src = M - 1 - k;
        energy_out[k] = c.op->center +
                        c.op->half_width * std::cos(M_PI * (double(src) + 0.5) / double(M));
        if (!bastin)
            for (int comp = 0; comp < 6; ++comp)
                sigma_out[k * 6 + comp] = prefactor * Kh[2 * (size_t(src) * 6 + comp)] / double(R);
    }
    if (bastin) {
        // sigma(mu, T = 0): cumulative trapezoid of Re(i zeta(eps)) over the
        // ascending Chebyshev grid (fftcheb_transport.hpp:635-659), zeta the
        // sample-averaged kernel.
        double running[6] = {0, 0, 0, 0, 0, 0}, prev[6] = {0, 0, 0, 0, 0, 0};
        double eps_prev = 0.0;
        for (int k = 0; k < M; ++k) {
            const int src = M - 1 - k;
            const double eps = std::cos(M_PI * (double(src) + 0.5) / double(M));
            for (int comp = 0; comp < 6; ++comp) {
                const double integrand = -Kh[2 * (size_t(src) * 6 + comp) + 1] / double(R);
                if (k > 0) running[comp] += 0.5 * (prev[comp] + integrand) * (eps - eps_prev);
                sigma_out[k * 6 + comp] = prefactor * running[comp];
                prev[comp] = integrand;
            }
            eps_prev = eps;
        }
    }
    if (stats) {
        stats->sections = n_sections;
        stats->fft_chunks = chunks;
        stats->recurrence_ms = rec_ms;
        stats->transform_ms = dct_ms;
        stats->store_bytes = 2 * size_t(M) * slot * cplx;
    }
    return RSATB_SUCCESS;
}

// ------------------------------------------------------------ QE route
//
// Quasi-eigenstate Greenwood (dc_spectrum_qe, fftcheb_transport.hpp:
// 662-884): the same bilinear form as the fftcheb Greenwood route,
// sigma(e_j) = sum_{m,m'} w_m(j) w_m'(j) <L_m|R_m'> / max(1e-14, 1 - e_j^2),
// w_m(j) = (m ? 2 : 1) g_m / pi T_m(e_j), evaluated at a window of nodes j
// only.  The weights are real, so it factors as <P_j|Q_j> with the left and
// right quasi-eigenstates P_j = sum_m w_m(j) L_m and Q_j = sum_m w_m(j) R_m:
// each pass adds a batch of QE_BATCH consecutive moment panels into all the
// node vectors in one launch (each node vector read and written once per
// batch, FP64 whatever the panel precision), and one fixed-order dot per
// (node, axis) finishes.  No row store and no transform.

constexpr int kQeBatch = 8;

template <typename T>
struct QePanels {
    const T* p[3 * kQeBatch];  // right: one [row][axis][sample] panel per
                               // moment; left: three [row][sample] per moment
};

// Q[j][a][row][s] += sum_b w[b][j] X_b(a, row, s) for the nb moments of a
// batch; one thread per (a, row, s).
template <typename T, bool RIGHT>
__global__ void qe_accumulate(int64_t n_rows, int R, int nb, int NE, QePanels<T> X,
                              const double* __restrict__ w, double2* __restrict__ Q) {
    const int64_t n_el = 3 * n_rows * R;
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n_el;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = e % R;
        const int64_t t = e / R;
        const int64_t row = t % n_rows;
        const int a = int(t / n_rows);
        double xr[kQeBatch], xi[kQeBatch];
#pragma unroll
        for (int b = 0; b < kQeBatch; ++b) {
            xr[b] = xi[b] = 0.0;
            if (b < nb) {
                const T* src = RIGHT ? X.p[b] + 2 * ((row * 3 + a) * R + s)
                                     : X.p[3 * b + a] + 2 * (row * R + s);
                xr[b] = double(src[0]);
                xi[b] = double(src[1]);
            }
        }
        for (int j = 0; j < NE; ++j) {
            double2 q = Q[int64_t(j) * n_el + e];
#pragma unroll
            for (int b = 0; b < kQeBatch; ++b) {
                if (b < nb) {
                    const double wb = __ldg(w + b * NE + j);
                    q.x = fma(wb, xr[b], q.x);
                    q.y = fma(wb, xi[b], q.y);
                }
            }
            Q[int64_t(j) * n_el + e] = q;
        }
    }
}

// D[j][a] = sum_{row, s} conj(P[j][a][row][s]) Q[j][a][row][s]: one CTA per
// (node, axis), fixed-order tree reduction.
__global__ void __launch_bounds__(256) qe_node_dots(int64_t per_axis, const double2* P,
                                                    const double2* Q, double* D) {
    __shared__ double red[2][256];
    const int64_t base = int64_t(blockIdx.x) * per_axis;
    double ar = 0.0, ai = 0.0;
    for (int64_t q = threadIdx.x; q < per_axis; q += blockDim.x) {
        const double2 x = P[base + q], y = Q[base + q];
        ar += x.x * y.x + x.y * y.y;
        ai += x.x * y.y - x.y * y.x;
    }
    red[0][threadIdx.x] = ar;
    red[1][threadIdx.x] = ai;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[0][threadIdx.x] += red[0][threadIdx.x + w];
            red[1][threadIdx.x] += red[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        D[2 * blockIdx.x] = red[0][0];
        D[2 * blockIdx.x + 1] = red[1][0];
    }
}

template <typename T>
int qe_impl(const Ctx& c, const rsatb_bsr_matrix* const* V, const T* psi, int R, int M,
            const std::vector<int>& nodes, double prefactor, int kernel, double* sigma_out,
            double* energy_out) {
    rsatb_context* ctx = c.ctx;
    cudaStream_t st = ctx->stream;
    const int b = c.op->H->block_size;
    const int nbr = c.op->H->n_block_rows;
    const int64_t N = int64_t(nbr) * b;
    const int W1 = 2 * R, W3 = 6 * R;
    const size_t cplx = 2 * sizeof(T);
    const int NE = int(nodes.size());
    const int RB = kQeBatch + 2;  // right ring: the batch plus the recurrence's predecessors

    std::vector<double> g(M);
    kpm_kernel_weights(kernel, M, g.data());
    // weights w[m][j] and the node energies (src = M - 1 - ascending index)
    std::vector<double> wts(size_t(M) * NE), denom(NE);
    for (int j = 0; j < NE; ++j) {
        const int src = M - 1 - nodes[j];
        const double th = M_PI * (double(src) + 0.5) / double(M);
        const double e = std::cos(th);
        denom[j] = std::max(1e-14, 1.0 - e * e);
        for (int m = 0; m < M; ++m)
            wts[size_t(m) * NE + j] = (m == 0 ? 1.0 : 2.0) * g[m] / M_PI * std::cos(double(m) * th);
    }
    DevBuf bW, bJ, bR, bL, bLA, bU, bWs, bQ, bP, bD;
    RSATB_TRY(bW.alloc(wts.size() * sizeof(double)));
    RSATB_CUDA_TRY(cudaMemcpyAsync(bW.p, wts.data(), wts.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, st));
    RSATB_TRY(bJ.alloc(size_t(N) * 3 * R * cplx));
    RSATB_TRY(bR.alloc(size_t(RB) * N * 3 * R * cplx));
    RSATB_TRY(bL.alloc(size_t(3) * N * R * cplx));
    RSATB_TRY(bLA.alloc(size_t(kQeBatch) * 3 * N * R * cplx));
    if (c.sandwich) {
        RSATB_TRY(bU.alloc(size_t(N) * 3 * R * cplx));
        RSATB_TRY(bWs.alloc(size_t(N) * 3 * R * cplx));
    }
    const int64_t n_el = 3 * N * R;
    RSATB_TRY(bQ.alloc(size_t(NE) * n_el * sizeof(double2)));
    RSATB_TRY(bP.alloc(size_t(NE) * n_el * sizeof(double2)));
    RSATB_TRY(bD.alloc(size_t(NE) * 3 * sizeof(double2)));
    RSATB_CUDA_TRY(cudaMemsetAsync(bQ.p, 0, size_t(NE) * n_el * sizeof(double2), st));
    RSATB_CUDA_TRY(cudaMemsetAsync(bP.p, 0, size_t(NE) * n_el * sizeof(double2), st));
    T* J[3];
    for (int a = 0; a < 3; ++a) J[a] = bJ.as<T>() + size_t(a) * N * 2 * R;
    auto rslot = [&](int m) { return bR.as<T>() + size_t(m % RB) * N * 6 * R; };
    T* l[3];
    for (int i = 0; i < 3; ++i) l[i] = bL.as<T>() + size_t(i) * N * 2 * R;
    auto laslot = [&](int bidx, int a) {
        return bLA.as<T>() + (size_t(bidx) * 3 + a) * N * 2 * R;
    };
    const unsigned grid = grid_for(n_el, ctx->sm_count);
    auto flush = [&](bool right, int m_last, int nb) -> int {
        QePanels<T> X{};
        const int m0 = m_last - nb + 1;
        for (int q = 0; q < nb; ++q) {
            if (right) {
                X.p[q] = rslot(m0 + q);
            } else {
                for (int a = 0; a < 3; ++a) X.p[3 * q + a] = laslot((m0 + q) % kQeBatch, a);
            }
        }
        const double* w = bW.as<double>() + size_t(m0) * NE;
        double2* dst = right ? bQ.as<double2>() : bP.as<double2>();
        if (right)
            qe_accumulate<T, true><<<grid, 256, 0, st>>>(N, R, nb, NE, X, w, dst);
        else
            qe_accumulate<T, false><<<grid, 256, 0, st>>>(N, R, nb, NE, X, w, dst);
        RSATB_LAUNCH_CHECK(ctx);
        return RSATB_SUCCESS;
    };

    // Right pass: R_0 = (J_a psi) packed [row][axis][sample], R_m by the
    // recurrence on the N x 3R panel.
    for (int a = 0; a < 3; ++a)
        RSATB_TRY(current_rows(c, V[a], W1, psi, J[a], 0, nbr, bU.p, bWs.p));
    pack_axes_kernel<T><<<grid_for(N * 3 * R, ctx->sm_count), 256, 0, st>>>(N, R, J[0], J[1],
                                                                           J[2], rslot(0));
    RSATB_LAUNCH_CHECK(ctx);
    for (int m = 0; m < M; ++m) {
        if (m == 1)
            RSATB_TRY(op_step(c, W3, rslot(0), nullptr, rslot(1), bU.p, bWs.p, 1.0, 0.0));
        else if (m >= 2)
            RSATB_TRY(op_step(c, W3, rslot(m - 1), rslot(m - 2), rslot(m), bU.p, bWs.p, 2.0,
                              -1.0));
        if ((m + 1) % kQeBatch == 0 || m == M - 1)
            RSATB_TRY(flush(true, m, m % kQeBatch + 1));
    }
    // Left pass: L_m = J_a T_m(Op) psi (J_a^H = J_a: V_a and the sandwich's
    // Z^H V_a Z are Hermitian).
    const T* lp = nullptr;
    const T* lc = psi;
    int li = 0;
    for (int m = 0; m < M; ++m) {
        if (m >= 1) {
            T* lo = l[li];
            li = (li + 1) % 3;
            if (m == 1) RSATB_TRY(op_step(c, W1, lc, nullptr, lo, bU.p, bWs.p, 1.0, 0.0));
            else RSATB_TRY(op_step(c, W1, lc, lp, lo, bU.p, bWs.p, 2.0, -1.0));
            lp = lc;
            lc = lo;
        }
        for (int a = 0; a < 3; ++a)
            RSATB_TRY(current_rows(c, V[a], W1, lc, laslot(m % kQeBatch, a), 0, nbr, bU.p,
                                   bWs.p));
        if ((m + 1) % kQeBatch == 0 || m == M - 1)
            RSATB_TRY(flush(false, m, m % kQeBatch + 1));
    }
    qe_node_dots<<<unsigned(NE * 3), 256, 0, st>>>(N * R, bP.as<double2>(), bQ.as<double2>(),
                                                  bD.as<double>());
    RSATB_LAUNCH_CHECK(ctx);
    std::vector<double> D(size_t(NE) * 6);
    RSATB_CUDA_TRY(cudaMemcpyAsync(D.data(), bD.p, D.size() * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    RSATB_CUDA_TRY(cudaStreamSynchronize(st));
    RSATB_TRY(ctx_check_fault(ctx));
    // Ascending energies (fftcheb_transport.hpp:940-954); sigma zero outside
    // the node window, Re of the sample-averaged kernel inside.
    for (int k = 0; k < M; ++k) {
        const int src = M - 1 - k;
        energy_out[k] = c.op->center +
                        c.op->half_width * std::cos(M_PI * (double(src) + 0.5) / double(M));
    }
    std::fill(sigma_out, sigma_out + size_t(M) * 6, 0.0);
    for (int j = 0; j < NE; ++j)
        for (int a = 0; a < 3; ++a) {
            const int comp = a == 0 ? 0 : (a == 1 ? 3 : 5);
            sigma_out[size_t(nodes[j]) * 6 + comp] =
                prefactor * D[2 * (size_t(j) * 3 + a)] / denom[j] / double(R);
        }
    return RSATB_SUCCESS;
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_dc_spectrum_fftcheb(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t Vx,
                                         rsatb_bsr_t Vy, rsatb_bsr_t Vz, const void* psi,
                                         int n_vectors, rsatb_dtype vec_dtype, int n_moments,
                                         int formulation, double prefactor,
                                         int partition_sections, size_t max_workspace_bytes,
                                         int kernel, double* sigma_out, double* energy_out,
                                         rsatb_fftcheb_stats* stats) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!op || !psi || !sigma_out || !energy_out)
        return set_error(RSATB_INVALID_ARGUMENT, "null argument");
    if (op->form != RSATB_FORM_ORTHOGONAL && op->form != RSATB_FORM_SANDWICH)
        return set_error(RSATB_NOT_SUPPORTED, "operator form %d is not available on the device",
                         op->form);
    const bool sandwich = op->form == RSATB_FORM_SANDWICH;
    const rsatb_bsr_matrix* mats[6] = {op->H, sandwich ? op->Z : op->H,
                                       sandwich ? op->ZH : op->H, Vx, Vy, Vz};
    const char* names[6] = {"H", "Z", "ZH", "Vx", "Vy", "Vz"};
    for (int i = 0; i < 6; ++i) {
        RSATB_TRY(check_bsr(mats[i], names[i]));
        if (mats[i]->n_block_rows != op->H->n_block_rows ||
            mats[i]->n_block_cols != op->H->n_block_rows ||
            mats[i]->block_size != op->H->block_size)
            return set_error(RSATB_INVALID_ARGUMENT, "%s does not match H's shape", names[i]);
        if (dtype_is_double(mats[i]->dtype) != dtype_is_double(vec_dtype))
            return set_error(RSATB_INVALID_ARGUMENT, "%s precision differs from the vectors'",
                             names[i]);
    }
    if (!dtype_is_complex(vec_dtype))
        return set_error(RSATB_INVALID_ARGUMENT, "transport needs complex sample vectors");
    if (!(op->half_width > 0.0))
        return set_error(RSATB_INVALID_ARGUMENT, "half_width must be positive");
    if (n_vectors <= 0 || n_moments <= 0)
        return set_error(RSATB_INVALID_ARGUMENT, "n_vectors and n_moments must be positive");
    if (6 * n_vectors > 1536)
        return set_error(RSATB_NOT_SUPPORTED, "%d samples exceed one block (256 at most)",
                         n_vectors);
    if (formulation != 0 && formulation != 1)
        return set_error(RSATB_INVALID_ARGUMENT,
                         "formulation %d: 0 (Greenwood) or 1 (Bastin)", formulation);
    if (!aligned16(psi)) return set_error(RSATB_INVALID_ARGUMENT, "psi must be 16-byte aligned");
    if (stats) *stats = rsatb_fftcheb_stats{};
    const rsatb_bsr_matrix* V[3] = {Vx, Vy, Vz};
    Ctx c{ctx, op, sandwich, int(vec_dtype)};
    if (dtype_is_double(vec_dtype))
        return fftcheb_impl<double>(c, V, static_cast<const double*>(psi), n_vectors, n_moments,
                                    formulation, prefactor, partition_sections,
                                    max_workspace_bytes, kernel, sigma_out, energy_out, stats);
    return fftcheb_impl<float>(c, V, static_cast<const float*>(psi), n_vectors, n_moments,
                               formulation, prefactor, partition_sections, max_workspace_bytes,
                               kernel, sigma_out, energy_out, stats);
}

extern "C" int rsatb_dc_spectrum_qe(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t Vx,
                                    rsatb_bsr_t Vy, rsatb_bsr_t Vz, const void* psi,
                                    int n_vectors, rsatb_dtype vec_dtype, int n_moments,
                                    double prefactor, int kernel, const int32_t* nodes,
                                    int n_nodes, double* sigma_out, double* energy_out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!op || !psi || !sigma_out || !energy_out || (n_nodes > 0 && !nodes))
        return set_error(RSATB_INVALID_ARGUMENT, "null argument");
    if (op->form != RSATB_FORM_ORTHOGONAL && op->form != RSATB_FORM_SANDWICH)
        return set_error(RSATB_NOT_SUPPORTED, "operator form %d is not available on the device",
                         op->form);
    const bool sandwich = op->form == RSATB_FORM_SANDWICH;
    const rsatb_bsr_matrix* mats[6] = {op->H, sandwich ? op->Z : op->H,
                                       sandwich ? op->ZH : op->H, Vx, Vy, Vz};
    const char* names[6] = {"H", "Z", "ZH", "Vx", "Vy", "Vz"};
    for (int i = 0; i < 6; ++i) {
        RSATB_TRY(check_bsr(mats[i], names[i]));
        if (mats[i]->n_block_rows != op->H->n_block_rows ||
            mats[i]->n_block_cols != op->H->n_block_rows ||
            mats[i]->block_size != op->H->block_size)
            return set_error(RSATB_INVALID_ARGUMENT, "%s does not match H's shape", names[i]);
        if (dtype_is_double(mats[i]->dtype) != dtype_is_double(vec_dtype))
            return set_error(RSATB_INVALID_ARGUMENT, "%s precision differs from the vectors'",
                             names[i]);
    }
    if (!dtype_is_complex(vec_dtype))
        return set_error(RSATB_INVALID_ARGUMENT, "transport needs complex sample vectors");
    if (!(op->half_width > 0.0))
        return set_error(RSATB_INVALID_ARGUMENT, "half_width must be positive");
    if (n_vectors <= 0 || n_moments <= 0)
        return set_error(RSATB_INVALID_ARGUMENT, "n_vectors and n_moments must be positive");
    if (6 * n_vectors > 1536)
        return set_error(RSATB_NOT_SUPPORTED, "%d samples exceed one block (256 at most)",
                         n_vectors);
    if (!aligned16(psi)) return set_error(RSATB_INVALID_ARGUMENT, "psi must be 16-byte aligned");
    // The node window: ascending output-grid indices, sorted and unique;
    // empty means every node (dc_spectrum_qe's nodes_ascending).
    std::vector<int> nd;
    if (n_nodes <= 0) {
        nd.resize(n_moments);
        for (int k = 0; k < n_moments; ++k) nd[k] = k;
    } else {
        nd.assign(nodes, nodes + n_nodes);
        std::sort(nd.begin(), nd.end());
        nd.erase(std::unique(nd.begin(), nd.end()), nd.end());
        if (nd.front() < 0 || nd.back() >= n_moments)
            return set_error(RSATB_INVALID_ARGUMENT, "dc_spectrum_qe: node index out of range");
    }
    const rsatb_bsr_matrix* V[3] = {Vx, Vy, Vz};
    Ctx c{ctx, op, sandwich, int(vec_dtype)};
    if (dtype_is_double(vec_dtype))
        return qe_impl<double>(c, V, static_cast<const double*>(psi), n_vectors, n_moments, nd,
                               prefactor, kernel, sigma_out, energy_out);
    return qe_impl<float>(c, V, static_cast<const float*>(psi), n_vectors, n_moments, nd,
                          prefactor, kernel, sigma_out, energy_out);
}
