// rsatb_b200.hpp -- C++17 host layer over the C ABI of rsatb_b200.h.
//
// The shapes RSATB's calc layer is written against, on the B200 library:
//
//   vbcsr::BlockSpMat<T>       uniform-block BSR matrix on the device
//                              (vbcsr BlockSpMat: mult_dense, duplicate,
//                              adjoint for mult_dense_adjoint), move-only
//   vbcsr::DistMultiVector<T>  device N x R row-major multivector
//                              (num_vectors, local_rows, set_random, host
//                              copies), move-only
//   calc::ISQRTMPreconditioner<T>   the graph-local factor Z and Z^H
//                              (rsatb/calc/preconditioner.hpp:169-240,
//                              constructed from a ready factor as the
//                              reference's kBorrowFactor does)
//   calc::Chebyshev<T>         the rescaled operator: the Orthogonal
//                              (H, emin, emax), Sandwich (H, pre, Symmetric,
//                              emin, emax) and Solve (H, S, emin, emax)
//                              constructors of rsatb/calc/cheby.hpp:167-201,
//                              public center / half_width, apply_op,
//                              op_is_hermitian
//   calc::kpm_dos_moments(Chebyshev<T>&, const DistMultiVector<T>&, int)
//                              (rsatb/calc/dos.hpp:125-190)
//   calc::evaluate_kpm_density (rsatb/calc/kpm.hpp:206-241)
//
// T is the element type of matrices and multivectors alike: double, float,
// std::complex<double> or std::complex<float>.  Errors surface as
// rsatb_b200::Error (a std::runtime_error carrying the C status), the way
// the reference's API level throws std::runtime_error on misconfiguration;
// the C ABI below never throws.  Every object keeps a reference to the
// Context it was made on; one host thread at a time per Context.
#ifndef RSATB_B200_HPP
#define RSATB_B200_HPP

#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "rsatb_b200.h"

namespace rsatb_b200 {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

inline void check(int status) {
    if (status != RSATB_SUCCESS) throw Error(status, rsatb_last_error());
}

template <typename T>
struct dtype_of;
template <>
struct dtype_of<double> {
    static constexpr rsatb_dtype value = RSATB_F64;
};
template <>
struct dtype_of<float> {
    static constexpr rsatb_dtype value = RSATB_F32;
};
template <>
struct dtype_of<std::complex<double>> {
    static constexpr rsatb_dtype value = RSATB_C128;
};
template <>
struct dtype_of<std::complex<float>> {
    static constexpr rsatb_dtype value = RSATB_C64;
};

// One device and its stream (rsatb_ctx_create / rsatb_ctx_destroy).
class Context {
public:
    explicit Context(int device = 0) { check(rsatb_ctx_create(device, &h_)); }
    ~Context() {
        if (h_) rsatb_ctx_destroy(h_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    rsatb_ctx_t handle() const { return h_; }
    void synchronize() const { check(rsatb_ctx_synchronize(h_)); }

private:
    rsatb_ctx_t h_ = nullptr;
};

namespace vbcsr {

template <typename T>
class DistMultiVector {
public:
    DistMultiVector(Context& ctx, int64_t local_rows, int num_vectors)
        : ctx_(&ctx), rows_(local_rows), cols_(num_vectors) {
        if (local_rows < 0 || num_vectors <= 0)
            throw Error(RSATB_INVALID_ARGUMENT, "DistMultiVector: bad shape");
        check(rsatb_device_alloc(ctx.handle(), bytes(), &data_));
    }
    ~DistMultiVector() {
        if (data_) rsatb_device_free(ctx_->handle(), data_);
    }
    DistMultiVector(DistMultiVector&& o) noexcept
        : ctx_(o.ctx_), rows_(o.rows_), cols_(o.cols_), data_(std::exchange(o.data_, nullptr)) {}
    DistMultiVector(const DistMultiVector&) = delete;
    DistMultiVector& operator=(const DistMultiVector&) = delete;

    int num_vectors() const { return cols_; }
    int64_t local_rows() const { return rows_; }
    size_t bytes() const { return size_t(rows_) * size_t(cols_) * sizeof(T); }
    void* data() { return data_; }
    const void* data() const { return data_; }
    Context& context() const { return *ctx_; }

    // SampleVectors::initialize's sample block (rsatb/calc/observables.hpp:
    // 84-96): seeded per (atom id, orbital, global column), Philox-4x32-10.
    void set_random(uint64_t seed, bool normalize, const std::vector<int64_t>& atom_index,
                    int orbitals_per_atom, rsatb_random_kind kind, int64_t first_column = 0) {
        check(rsatb_set_random(ctx_->handle(), seed, kind, normalize ? 1 : 0, atom_index.data(),
                               int(atom_index.size()), orbitals_per_atom, rows_, cols_,
                               first_column, dtype_of<T>::value, data_));
    }
    void copy_from_host(const std::vector<T>& h) {
        if (h.size() * sizeof(T) != bytes())
            throw Error(RSATB_INVALID_ARGUMENT, "copy_from_host: size differs");
        check(rsatb_copy_to_device(ctx_->handle(), data_, h.data(), bytes()));
    }
    std::vector<T> to_host() const {
        std::vector<T> h(size_t(rows_) * size_t(cols_));
        check(rsatb_copy_to_host_sync(ctx_->handle(), h.data(), data_, bytes()));
        return h;
    }

private:
    Context* ctx_;
    int64_t rows_;
    int cols_;
    void* data_ = nullptr;
};

template <typename T>
class BlockSpMat {
public:
    // construct + add_block + assemble of vbcsr in one step: block k of block
    // row i holds rows i*b.., columns col_ind[k]*b.. at values[k*b*b ..].
    BlockSpMat(Context& ctx, int n_block_rows, int n_block_cols, int block_size,
               const std::vector<int32_t>& row_ptr, const std::vector<int32_t>& col_ind,
               const std::vector<T>& values, unsigned flags = 0)
        : ctx_(&ctx) {
        if (row_ptr.size() != size_t(n_block_rows) + 1 ||
            values.size() != col_ind.size() * size_t(block_size) * size_t(block_size))
            throw Error(RSATB_INVALID_ARGUMENT, "BlockSpMat: array sizes differ from the shape");
        check(rsatb_bsr_create(ctx.handle(), n_block_rows, n_block_cols, block_size,
                               int64_t(col_ind.size()), row_ptr.data(), col_ind.data(),
                               values.data(), dtype_of<T>::value, flags, &h_));
    }
    ~BlockSpMat() {
        if (h_) rsatb_bsr_destroy(h_);
    }
    BlockSpMat(BlockSpMat&& o) noexcept : ctx_(o.ctx_), h_(std::exchange(o.h_, nullptr)) {}
    BlockSpMat(const BlockSpMat&) = delete;
    BlockSpMat& operator=(const BlockSpMat&) = delete;

    rsatb_bsr_t handle() const { return h_; }
    Context& context() const { return *ctx_; }
    int block_size() const { return info().block_size; }
    int64_t rows() const { return int64_t(info().n_block_rows) * info().block_size; }

    // Y = alpha * A X (vbcsr mult_dense).
    void mult_dense(const DistMultiVector<T>& X, DistMultiVector<T>& Y, double alpha = 1.0) const {
        check(rsatb_bsr_mult_dense(ctx_->handle(), h_, X.data(), Y.data(), X.num_vectors(),
                                   dtype_of<T>::value, alpha));
    }
    // A^H as a matrix of its own (what mult_dense_adjoint applies).
    BlockSpMat adjoint() const {
        rsatb_bsr_t out = nullptr;
        check(rsatb_bsr_adjoint(ctx_->handle(), h_, &out));
        return BlockSpMat(ctx_, out);
    }
    // Takes ownership of a matrix an entry point created (rsatb_inverse_sqrt_refine).
    static BlockSpMat adopt(Context& ctx, rsatb_bsr_t h) { return BlockSpMat(&ctx, h); }
    int64_t nnz_blocks() const { return info().nnz; }
    // Block row offsets and block columns (row_ptr, col_ind) on the host.
    void pattern(std::vector<int32_t>& row_ptr, std::vector<int32_t>& col_ind) const {
        const Info i = info();
        row_ptr.resize(size_t(i.n_block_rows) + 1);
        col_ind.resize(size_t(i.nnz));
        check(rsatb_bsr_pattern(ctx_->handle(), h_, row_ptr.data(), col_ind.data()));
    }

private:
    struct Info {
        int n_block_rows, n_block_cols, block_size;
        int64_t nnz;
        int dtype;
        unsigned flags;
    };
    BlockSpMat(Context* ctx, rsatb_bsr_t h) : ctx_(ctx), h_(h) {}
    Info info() const {
        Info i{};
        check(rsatb_bsr_info(h_, &i.n_block_rows, &i.n_block_cols, &i.block_size, &i.nnz,
                             &i.dtype, &i.flags));
        return i;
    }
    Context* ctx_;
    rsatb_bsr_t h_ = nullptr;
};

}  // namespace vbcsr

namespace calc {

using vbcsr::BlockSpMat;
using vbcsr::DistMultiVector;

enum class ChebyOpForm { Orthogonal, Sandwich, Solve };
enum class PreconditionerType { Left, Right, Symmetric };
enum class ChebyMode { NORMAL, ADJOINT };

// The graph-local factor Z of S^-1/2 with its adjoint built once on the
// device, so that the sandwich's Z^H x also runs as a forward row gather.
template <typename T>
class ISQRTMPreconditioner {
public:
    explicit ISQRTMPreconditioner(BlockSpMat<T>& Z) : Z_(&Z), ZH_(Z.adjoint()) {}
    const BlockSpMat<T>& Z() const { return *Z_; }
    const BlockSpMat<T>& ZH() const { return ZH_; }

private:
    BlockSpMat<T>* Z_;
    BlockSpMat<T> ZH_;
};

template <typename T>
class Chebyshev {
public:
    BlockSpMat<T>& H;
    BlockSpMat<T>* S = nullptr;
    ISQRTMPreconditioner<T>* M = nullptr;
    const ChebyOpForm form = ChebyOpForm::Orthogonal;
    double center = 0.0;
    double half_width = 1.0;
    double cg_tol = 1e-8;      // Solve form: the CG of every application
    int cg_max_iter = 1000;

    // Orthogonal: the recurrence iterates H.
    Chebyshev(BlockSpMat<T>& ham, double emin, double emax)
        : H(ham), form(ChebyOpForm::Orthogonal) {
        set_window(emin, emax);
    }
    // Sandwich: the recurrence iterates Z^H H Z (a Symmetric preconditioner
    // only, as in the reference).
    Chebyshev(BlockSpMat<T>& ham, ISQRTMPreconditioner<T>& pre, PreconditionerType type,
              double emin, double emax)
        : H(ham), M(&pre), form(ChebyOpForm::Sandwich) {
        if (type != PreconditionerType::Symmetric)
            throw Error(RSATB_INVALID_ARGUMENT,
                        "Chebyshev: the Z^H H Z sandwich needs a Symmetric preconditioner");
        set_window(emin, emax);
    }
    // Solve: the recurrence iterates S^-1 H, one CG with S per application.
    Chebyshev(BlockSpMat<T>& ham, BlockSpMat<T>& ovp, double emin, double emax)
        : H(ham), S(&ovp), form(ChebyOpForm::Solve) {
        set_window(emin, emax);
    }

    void set_window(double emin, double emax) {
        if (!(emax > emin))
            throw Error(RSATB_INVALID_ARGUMENT, "Chebyshev: the window needs emax > emin");
        center = 0.5 * (emax + emin);
        half_width = 0.5 * (emax - emin);
    }
    bool op_is_hermitian() const { return form != ChebyOpForm::Solve; }

    // Y = ((Op) X - center X) / half_width; the three forms are Hermitian or
    // served NORMAL only, so mode only matters for being refused.
    void apply_op(const DistMultiVector<T>& X, DistMultiVector<T>& Y,
                  ChebyMode mode = ChebyMode::NORMAL) const {
        if (form == ChebyOpForm::Solve && mode == ChebyMode::ADJOINT)
            throw Error(RSATB_NOT_SUPPORTED, "apply_op: the Solve form serves NORMAL only");
        const rsatb_cheb_op op = c_op();
        check(rsatb_cheb_apply_op(H.context().handle(), &op, X.data(), Y.data(),
                                  X.num_vectors(), dtype_of<T>::value));
    }

    // Y = sum_n c_n T_n(Op~) X, Chebyshev::propagate (rsatb/calc/cheby.hpp:
    // 367-441); a real panel takes Re(c_n).
    void propagate(const DistMultiVector<T>& X, DistMultiVector<T>& Y,
                   const std::vector<std::complex<double>>& coeffs) const {
        std::vector<double> c(2 * coeffs.size());
        for (size_t n = 0; n < coeffs.size(); ++n) {
            c[2 * n] = coeffs[n].real();
            c[2 * n + 1] = coeffs[n].imag();
        }
        const rsatb_cheb_op op = c_op();
        check(rsatb_cheb_propagate(H.context().handle(), &op, X.data(), Y.data(),
                                   X.num_vectors(), dtype_of<T>::value, c.data(),
                                   int(coeffs.size())));
    }
    // Y = scale * (V dressed by the form) X, Chebyshev::apply_dual
    // (rsatb/calc/cheby.hpp:249-291): V, Z^H V Z or S^-1 V (ADJOINT: V S^-1).
    void apply_dual(const BlockSpMat<T>& V, const DistMultiVector<T>& X, DistMultiVector<T>& Y,
                    double scale = 1.0, ChebyMode mode = ChebyMode::NORMAL) const {
        const rsatb_cheb_op op = c_op();
        if (mode == ChebyMode::ADJOINT)
            check(rsatb_cheb_apply_dual_adjoint(H.context().handle(), &op, V.handle(), X.data(),
                                                Y.data(), X.num_vectors(), dtype_of<T>::value,
                                                scale));
        else
            check(rsatb_cheb_apply_dual(H.context().handle(), &op, V.handle(), X.data(),
                                        Y.data(), X.num_vectors(), dtype_of<T>::value, scale));
    }
    // mu_n = <psi|T_n(Op~)|psi> averaged over the columns by the plain
    // recurrence, Chebyshev::compute_moments (rsatb/calc/cheby.hpp:479-514).
    std::vector<std::complex<double>> compute_moments(const DistMultiVector<T>& psi,
                                                      int n_moments) const {
        if (n_moments <= 0) return {};
        const rsatb_cheb_op op = c_op();
        std::vector<double> mu(2 * size_t(n_moments));
        check(rsatb_kpm_dos_moments(H.context().handle(), &op, psi.data(), psi.num_vectors(),
                                    dtype_of<T>::value, n_moments, 0, mu.data(), nullptr));
        std::vector<std::complex<double>> out(n_moments);
        for (int n = 0; n < n_moments; ++n) out[n] = {mu[2 * n], mu[2 * n + 1]};
        return out;
    }

    rsatb_cheb_op c_op() const {
        rsatb_cheb_op op{};
        op.form = form == ChebyOpForm::Sandwich ? RSATB_FORM_SANDWICH
                  : form == ChebyOpForm::Solve  ? RSATB_FORM_SOLVE
                                                : RSATB_FORM_ORTHOGONAL;
        op.H = H.handle();
        if (M) {
            op.Z = M->Z().handle();
            op.ZH = M->ZH().handle();
        }
        op.S = S ? S->handle() : nullptr;
        op.center = center;
        op.half_width = half_width;
        op.cg_tol = cg_tol;
        op.cg_max_iter = cg_max_iter;
        return op;
    }
};

// KPM moments averaged over psi's columns, two per application for the
// Hermitian forms (rsatb/calc/dos.hpp:125-190); the whole recurrence runs on
// the device.
template <typename T>
std::vector<std::complex<double>> kpm_dos_moments(Chebyshev<T>& cheby,
                                                  const DistMultiVector<T>& psi,
                                                  int n_moments) {
    if (n_moments <= 0) return {};
    const rsatb_cheb_op op = cheby.c_op();
    std::vector<double> mu(2 * size_t(n_moments));
    check(rsatb_kpm_dos_moments(cheby.H.context().handle(), &op, psi.data(),
                                psi.num_vectors(), dtype_of<T>::value, n_moments,
                                cheby.op_is_hermitian() ? 1 : 0, mu.data(), nullptr));
    std::vector<std::complex<double>> out(n_moments);
    for (int n = 0; n < n_moments; ++n) out[n] = {mu[2 * n], mu[2 * n + 1]};
    return out;
}

// Extreme eigenvalues of the operator cheby iterates, applied unscaled (its
// window is ignored), by Lanczos on the device: the PRIMME call of
// EstimateSpectralBounds (rsatb/setup/spectral_bounds.hpp:311-490).  The
// caller pads by |residual| and BoundsOptions::padding and applies the
// reference's fallback when converged == 0.
template <typename T>
rsatb_lanczos_result lanczos_extremes(const Chebyshev<T>& cheby, double tol = 1e-3,
                                      int max_matvecs = 10000, uint64_t seed = 2) {
    const rsatb_cheb_op op = cheby.c_op();
    rsatb_lanczos_options o{};
    o.tol = tol;
    o.max_matvecs = max_matvecs;
    o.seed = seed;
    rsatb_lanczos_result r{};
    check(rsatb_lanczos_extremes(cheby.H.context().handle(), &op, &o, &r));
    return r;
}

// rsatb::calc::inverse_sqrt (rsatb/calc/isqrtm.hpp:262) for a real FP64
// overlap from a seed factor Z0 (the graph-local S^-1/2): Newton-Schulz with
// block SpGEMMs, the drop threshold sptol and the reference's stopping rules.
struct InverseSqrtOptions {
    double tol = 1e-7;
    double sptol = 1e-6;
    int maxit = 20;
    int route = 0;  // 0: X reformed or propagated by cost, 1: always reformed
};
using InverseSqrtReport = rsatb_ns_refine_report;

inline BlockSpMat<double> inverse_sqrt(const BlockSpMat<double>& S, const BlockSpMat<double>& Z0,
                                       const InverseSqrtOptions& opts = {},
                                       InverseSqrtReport* report = nullptr) {
    rsatb_ns_refine_options o{};
    o.tol = opts.tol;
    o.sptol = opts.sptol;
    o.maxit = opts.maxit;
    o.route = opts.route;
    rsatb_ns_refine_report rep{};
    rsatb_bsr_t Z = nullptr;
    check(rsatb_inverse_sqrt_refine(S.context().handle(), S.handle(), Z0.handle(), &o, &Z, &rep));
    if (report) *report = rep;
    return BlockSpMat<double>::adopt(S.context(), Z);
}

// The DC spectrum by the FFT-Chebyshev method, rsatb::calc::
// dc_spectrum_fftcheb (rsatb/calc/fftcheb_transport.hpp:543): Vx, Vy, Vz
// the velocity matrices (H's shape and type), psi the complex samples.
// sigma_out receives n_moments x 6 (xx xy xz yy yz zz; Greenwood fills the
// diagonal) scaled by prefactor, energy_out the ascending energies.
enum class DCFormulation { Greenwood = 0, Bastin = 1 };

template <typename T>
void dc_spectrum_fftcheb(const Chebyshev<T>& cheby, const BlockSpMat<T>& Vx,
                         const BlockSpMat<T>& Vy, const BlockSpMat<T>& Vz,
                         const DistMultiVector<T>& psi, int n_moments,
                         DCFormulation formulation, double prefactor, int partition_sections,
                         size_t max_workspace_mb, std::vector<double>& sigma_out,
                         std::vector<double>& energy_out,
                         rsatb_kpm_kernel kernel = RSATB_KPM_JACKSON) {
    static_assert(dtype_of<T>::value == RSATB_C128 || dtype_of<T>::value == RSATB_C64,
                  "dc_spectrum_fftcheb takes complex sample vectors");
    const rsatb_cheb_op op = cheby.c_op();
    sigma_out.assign(6 * size_t(n_moments), 0.0);
    energy_out.assign(size_t(n_moments), 0.0);
    check(rsatb_dc_spectrum_fftcheb(cheby.H.context().handle(), &op, Vx.handle(), Vy.handle(),
                                    Vz.handle(), psi.data(), psi.num_vectors(),
                                    dtype_of<T>::value, n_moments, int(formulation), prefactor,
                                    partition_sections, max_workspace_mb << 20, kernel,
                                    sigma_out.data(), energy_out.data(), nullptr));
}

// rho(x_j) from the moments with the Jackson (or another) kernel
// (rsatb/calc/kpm.hpp:206-241), x clamped by edge_inset.
inline std::vector<double> evaluate_kpm_density(Context& ctx,
                                                const std::vector<std::complex<double>>& mu,
                                                const std::vector<double>& x,
                                                double edge_inset = 1e-3,
                                                rsatb_kpm_kernel kernel = RSATB_KPM_JACKSON) {
    std::vector<double> m(2 * mu.size()), rho(x.size());
    for (size_t n = 0; n < mu.size(); ++n) {
        m[2 * n] = mu[n].real();
        m[2 * n + 1] = mu[n].imag();
    }
    check(rsatb_evaluate_kpm_density(ctx.handle(), m.data(), int(mu.size()), x.data(),
                                     int(x.size()), edge_inset, kernel, rho.data()));
    return rho;
}

}  // namespace calc
}  // namespace rsatb_b200

#endif  // RSATB_B200_HPP
