// A C++17 program that computes a Kubo-Greenwood spectrum the way a
// reference caller (ComputeDcSpectrum -> dc_spectrum_fftcheb) would, through
// include/rsatb_b200.hpp: Chebyshev<std::complex<double>> on H and the three
// velocity matrices V_a = i W_a as complex BlockSpMats.
//
// Usage: transport_consumer <input file>
// The input (native-endian binary) holds
//   int32  n_block_rows, block_size, nnz_blocks, n_vectors, n_moments, formulation
//   f64    emin, emax
//   int32  row_ptr[n_block_rows + 1], col_ind[nnz_blocks]
//   f64    H values, then W_x, W_y, W_z values (real, nnz_blocks * b * b each)
//   f64    psi[rows * n_vectors] as (re, im) pairs, row-major
// and the program prints sigma (n_moments x 6) and the energies as JSON.
#include <cstdio>
#include <fstream>
#include <vector>

#include "rsatb_b200.hpp"

namespace {

template <typename X>
void read(std::ifstream& in, X* dst, size_t n) {
    in.read(reinterpret_cast<char*>(dst), std::streamsize(n * sizeof(X)));
    if (!in) throw std::runtime_error("truncated input");
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
        double window[2];
        read(in, hdr, 6);
        read(in, window, 2);
        const int nbr = hdr[0], b = hdr[1], nnz = hdr[2], R = hdr[3], M = hdr[4],
                  formulation = hdr[5];
        std::vector<int32_t> row_ptr(static_cast<size_t>(nbr) + 1);
        std::vector<int32_t> col_ind(static_cast<size_t>(nnz));
        read(in, row_ptr.data(), row_ptr.size());
        read(in, col_ind.data(), col_ind.size());
        const size_t nv = size_t(nnz) * b * b;
        std::vector<double> hv(nv), w[3] = {std::vector<double>(nv), std::vector<double>(nv),
                                            std::vector<double>(nv)};
        read(in, hv.data(), nv);
        for (auto& x : w) read(in, x.data(), nv);
        const int64_t n_rows = int64_t(nbr) * b;
        std::vector<cd> ph(static_cast<size_t>(n_rows) * R);
        read(in, reinterpret_cast<double*>(ph.data()), 2 * ph.size());

        std::vector<cd> hc(nv), vc[3] = {std::vector<cd>(nv), std::vector<cd>(nv),
                                         std::vector<cd>(nv)};
        for (size_t i = 0; i < nv; ++i) {
            hc[i] = cd(hv[i], 0.0);
            for (int a = 0; a < 3; ++a) vc[a][i] = cd(0.0, w[a][i]);  // V_a = i W_a
        }
        Context ctx(0);
        vbcsr::BlockSpMat<cd> H(ctx, nbr, nbr, b, row_ptr, col_ind, hc);
        vbcsr::BlockSpMat<cd> Vx(ctx, nbr, nbr, b, row_ptr, col_ind, vc[0]);
        vbcsr::BlockSpMat<cd> Vy(ctx, nbr, nbr, b, row_ptr, col_ind, vc[1]);
        vbcsr::BlockSpMat<cd> Vz(ctx, nbr, nbr, b, row_ptr, col_ind, vc[2]);
        vbcsr::DistMultiVector<cd> psi(ctx, n_rows, R);
        psi.copy_from_host(ph);
        calc::Chebyshev<cd> cheby(H, window[0], window[1]);
        std::vector<double> sigma, energy;
        calc::dc_spectrum_fftcheb(cheby, Vx, Vy, Vz, psi, M,
                                  formulation ? calc::DCFormulation::Bastin
                                              : calc::DCFormulation::Greenwood,
                                  1.0, 0, 0, sigma, energy);
        std::printf("{\"sigma\": [");
        for (size_t i = 0; i < sigma.size(); ++i) std::printf("%s%.17g", i ? ", " : "", sigma[i]);
        std::printf("], \"energy\": [");
        for (size_t i = 0; i < energy.size(); ++i)
            std::printf("%s%.17g", i ? ", " : "", energy[i]);
        std::printf("]}\n");
    } catch (const Error& e) {
        std::fprintf(stderr, "rsatb error %d: %s\n", e.status(), e.what());
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
