// A second C++17 program against RSATB's calc-layer shapes, through
// include/rsatb_b200.hpp: Chebyshev<double>::propagate, apply_dual and
// compute_moments, the spectral-bounds Lanczos and the sparse inverse_sqrt
// refinement, as a reference caller (time propagation, transport currents,
// EstimateSpectralBounds, build_preconditioner) would drive them.
//
// Usage: calc_consumer <input file>
// The input (native-endian binary) holds
//   int32  n_block_rows, block_size, nnz_blocks, n_vectors, n_coeffs, n_moments
//   f64    emin, emax, scale
//   u64    seed
//   int32  row_ptr[n_block_rows + 1], col_ind[nnz_blocks]
//   f64    H, V, S, Z0 values (nnz_blocks * b * b each, one shared pattern)
//   f64    coeffs[2 * n_coeffs] as (re, im)
// and the program prints one JSON line with the results.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <numeric>
#include <vector>

#include "rsatb_b200.hpp"

namespace {

template <typename X>
void read(std::ifstream& in, X* dst, size_t n) {
    in.read(reinterpret_cast<char*>(dst), std::streamsize(n * sizeof(X)));
    if (!in) throw std::runtime_error("truncated input");
}

void print_array(const char* name, const std::vector<double>& v, bool last = false) {
    std::printf("\"%s\": [", name);
    for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i]);
    std::printf("]%s", last ? "" : ", ");
}

}  // namespace

int main(int argc, char** argv) {
    using namespace rsatb_b200;
    using cd = std::complex<double>;
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <input file>\n", argv[0]);
        return 2;
    }
    try {
        std::ifstream in(argv[1], std::ios::binary);
        if (!in) throw std::runtime_error("cannot open input");
        int32_t hdr[6];
        double par[3];
        uint64_t seed = 0;
        read(in, hdr, 6);
        read(in, par, 3);
        read(in, &seed, 1);
        const int nbr = hdr[0], b = hdr[1], nnz = hdr[2], R = hdr[3], n_coeffs = hdr[4],
                  n_moments = hdr[5];
        std::vector<int32_t> row_ptr(size_t(nbr) + 1);
        std::vector<int32_t> col_ind(static_cast<size_t>(nnz));
        read(in, row_ptr.data(), row_ptr.size());
        read(in, col_ind.data(), col_ind.size());
        const size_t nv = size_t(nnz) * b * b;
        std::vector<double> hv(nv), vv(nv), sv(nv), zv(nv), cr(2 * size_t(n_coeffs));
        read(in, hv.data(), nv);
        read(in, vv.data(), nv);
        read(in, sv.data(), nv);
        read(in, zv.data(), nv);
        read(in, cr.data(), cr.size());

        Context ctx(0);
        vbcsr::BlockSpMat<double> H(ctx, nbr, nbr, b, row_ptr, col_ind, hv);
        vbcsr::BlockSpMat<double> V(ctx, nbr, nbr, b, row_ptr, col_ind, vv);
        vbcsr::BlockSpMat<double> S(ctx, nbr, nbr, b, row_ptr, col_ind, sv);
        vbcsr::BlockSpMat<double> Z0(ctx, nbr, nbr, b, row_ptr, col_ind, zv);
        const int64_t n_rows = int64_t(nbr) * b;
        vbcsr::DistMultiVector<double> psi(ctx, n_rows, R), Y(ctx, n_rows, R);
        std::vector<int64_t> atoms(static_cast<size_t>(nbr));
        std::iota(atoms.begin(), atoms.end(), 0);
        psi.set_random(seed, true, atoms, b, RSATB_RANDOM_RADEMACHER);

        calc::Chebyshev<double> cheby(H, par[0], par[1]);
        std::vector<cd> coeffs(static_cast<size_t>(n_coeffs));
        for (int n = 0; n < n_coeffs; ++n) coeffs[n] = {cr[2 * n], cr[2 * n + 1]};

        std::printf("{");
        // Spectral bounds of H (its extreme Ritz pairs to 1e-8).
        const rsatb_lanczos_result lr = calc::lanczos_extremes(cheby, 1e-8, 400);
        print_array("lanczos", {lr.theta_min, lr.theta_max, lr.res_min, lr.res_max,
                                double(lr.matvecs), double(lr.converged)});
        // Y = sum c_n T_n(H~) psi
        cheby.propagate(psi, Y, coeffs);
        print_array("propagate", Y.to_host());
        // Y = scale V psi (the Orthogonal form's dual)
        cheby.apply_dual(V, psi, Y, par[2]);
        print_array("apply_dual", Y.to_host());
        // plain-recurrence moments
        const std::vector<cd> mu = cheby.compute_moments(psi, n_moments);
        std::vector<double> mre(mu.size());
        for (size_t n = 0; n < mu.size(); ++n) mre[n] = mu[n].real();
        print_array("moments", mre);

        // Z = S^-1/2 refined from the seed; ||Z^T S Z psi - psi|| / ||psi||.
        calc::InverseSqrtOptions opts;
        opts.tol = 1e-10;
        opts.sptol = 0.0;
        opts.route = 1;
        calc::InverseSqrtReport rep{};
        vbcsr::BlockSpMat<double> Z = calc::inverse_sqrt(S, Z0, opts, &rep);
        vbcsr::BlockSpMat<double> ZT = Z.adjoint();
        vbcsr::DistMultiVector<double> u(ctx, n_rows, R), w(ctx, n_rows, R);
        Z.mult_dense(psi, u);
        S.mult_dense(u, w);
        ZT.mult_dense(w, u);
        const std::vector<double> out = u.to_host(), ref = psi.to_host();
        double num = 0.0, den = 0.0;
        for (size_t i = 0; i < out.size(); ++i) {
            num += (out[i] - ref[i]) * (out[i] - ref[i]);
            den += ref[i] * ref[i];
        }
        std::vector<int32_t> zrp, zci;
        Z.pattern(zrp, zci);
        print_array("refine", {double(rep.steps), double(rep.converged), rep.residual,
                               double(Z.nnz_blocks()), double(zci.size()),
                               std::sqrt(num / den)},
                    true);
        std::printf("}\n");
    } catch (const Error& e) {
        std::fprintf(stderr, "rsatb error %d: %s\n", e.status(), e.what());
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
