// A C++17 program written against RSATB's calc-layer shapes, built on the
// rsatb_b200 C ABI through include/rsatb_b200.hpp: the way a reference
// caller (ComputeDos -> kpm_dos_moments) would drive the B200 library.
//
// Usage: kpm_consumer <input file>
// The input (native-endian binary) holds
//   int32  n_block_rows, block_size, nnz_blocks, has_z, n_vectors, n_moments,
//          orbitals_per_atom
//   f64    emin, emax
//   u64    seed
//   int32  row_ptr[n_block_rows + 1], col_ind[nnz_blocks]
//   f64    H values[nnz_blocks * b * b], then (has_z) Z values, same pattern
// It builds H (and the sandwich Z^H H Z when has_z), draws n_vectors
// Rademacher sample vectors, runs kpm_dos_moments(Chebyshev&, psi,
// n_moments) and prints the moments as one JSON line.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>
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
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <input file>\n", argv[0]);
        return 2;
    }
    try {
        std::ifstream in(argv[1], std::ios::binary);
        if (!in) throw std::runtime_error("cannot open input");
        int32_t hdr[7];
        double window[2];
        uint64_t seed = 0;
        read(in, hdr, 7);
        read(in, window, 2);
        read(in, &seed, 1);
        const int nbr = hdr[0], b = hdr[1], nnz = hdr[2], has_z = hdr[3], R = hdr[4],
                  n_moments = hdr[5], orbitals = hdr[6];
        std::vector<int32_t> row_ptr(size_t(nbr) + 1);
        std::vector<int32_t> col_ind(static_cast<size_t>(nnz));
        std::vector<double> hv(size_t(nnz) * b * b), zv;
        read(in, row_ptr.data(), row_ptr.size());
        read(in, col_ind.data(), col_ind.size());
        read(in, hv.data(), hv.size());
        if (has_z) {
            zv.resize(hv.size());
            read(in, zv.data(), zv.size());
        }

        Context ctx(0);
        vbcsr::BlockSpMat<double> H(ctx, nbr, nbr, b, row_ptr, col_ind, hv);
        const int64_t n_rows = int64_t(nbr) * b;
        vbcsr::DistMultiVector<double> psi(ctx, n_rows, R);
        std::vector<int64_t> atoms(size_t(n_rows / orbitals));
        std::iota(atoms.begin(), atoms.end(), 0);
        psi.set_random(seed, true, atoms, orbitals, RSATB_RANDOM_RADEMACHER);

        std::vector<std::complex<double>> mu;
        if (has_z) {
            vbcsr::BlockSpMat<double> Z(ctx, nbr, nbr, b, row_ptr, col_ind, zv);
            calc::ISQRTMPreconditioner<double> pre(Z);
            calc::Chebyshev<double> cheby(H, pre, calc::PreconditionerType::Symmetric, window[0],
                                          window[1]);
            mu = calc::kpm_dos_moments(cheby, psi, n_moments);
        } else {
            calc::Chebyshev<double> cheby(H, window[0], window[1]);
            mu = calc::kpm_dos_moments(cheby, psi, n_moments);
        }
        std::printf("{\"moments_re\": [");
        for (size_t n = 0; n < mu.size(); ++n)
            std::printf("%s%.17g", n ? ", " : "", mu[n].real());
        std::printf("], \"moments_im\": [");
        for (size_t n = 0; n < mu.size(); ++n)
            std::printf("%s%.17g", n ? ", " : "", mu[n].imag());
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
