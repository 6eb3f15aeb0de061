// Check program for the C++20 drop-in classes of include/loki_b200.hpp: the
// reference's FFACUDA<float> / PulsarSearchConfig / compute_ffa_scores_cuda
// interface, implemented over the C ABI.
//
//   ffacuda_check <input.bin> <fold.bin> <scores.bin> <cfold.bin> <cscores.bin>
//
// input.bin: uint64 nsamps, double tsamp, uint64 nbins, double eta, uint32
// nparams, double limits[2 * nparams], uint32 nwidths, uint32 widths[nwidths],
// float ts_e[nsamps], float ts_v[nsamps]. Writes the final fold of
// FFACUDA<float>::execute (host spans) and the scores of
// compute_ffa_scores_cuda with use_fourier = false, then the final complex
// fold of FFACUDA<ComplexTypeCUDA>::execute and the scores of
// compute_ffa_scores_cuda with use_fourier = true (the default). Exit status
// 0 when every check passed.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "loki_b200.hpp"

namespace {

using loki_b200::SizeType;

template <class T> T read_one(std::ifstream& in) {
    T v{};
    in.read(reinterpret_cast<char*>(&v), sizeof(T));
    return v;
}

template <class T> std::vector<T> read_n(std::ifstream& in, std::size_t n) {
    std::vector<T> v(n);
    in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
    return v;
}

template <class T> void write_all(const char* path, const std::vector<T>& v) {
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

SizeType plan_nbins_f(SizeType nbins) { return nbins / 2 + 1; }

}  // namespace

int main(int argc, char** argv) {
    using namespace loki_b200;
    if (argc != 6) {
        std::cerr << "usage: ffacuda_check <input.bin> <fold.bin> <scores.bin> <cfold.bin> <cscores.bin>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    const auto nsamps = read_one<uint64_t>(in);
    const auto tsamp = read_one<double>(in);
    const auto nbins = read_one<uint64_t>(in);
    const auto eta = read_one<double>(in);
    const auto np = read_one<uint32_t>(in);
    const auto lim = read_n<double>(in, 2 * np);
    const auto nw = read_one<uint32_t>(in);
    const auto w32 = read_n<uint32_t>(in, nw);
    const auto ts_e = read_n<float>(in, nsamps);
    const auto ts_v = read_n<float>(in, nsamps);
    if (!in) {
        std::cerr << "short input\n";
        return 2;
    }
    std::vector<ParamLimit> limits(np);
    for (uint32_t i = 0; i < np; ++i) {
        limits[i] = {lim[2 * i], lim[2 * i + 1]};
    }
    const std::vector<SizeType> widths(w32.begin(), w32.end());
    try {
        const search::PulsarSearchConfig cfg(nsamps, tsamp, nbins, eta, limits, 0.2, 1.5,
                                             /*use_fourier=*/false, 1, std::nullopt, std::nullopt, 5.0,
                                             widths);
        const search::PulsarSearchConfig copy = cfg;  // copyable, like the reference's
        algorithms::FFACUDA<float> ffa(copy);
        algorithms::FFACUDA<float> moved = std::move(ffa);  // move-only PIMPL
        std::vector<float> fold(moved.get_plan().get_fold_size());
        moved.execute(ts_e, ts_v, fold);
        write_all(argv[2], fold);
        auto [scores, plan] = algorithms::compute_ffa_scores_cuda(ts_e, ts_v, cfg);
        if (scores.size() != plan.get_ncoords_final() * widths.size()) {
            std::cerr << "scores size mismatch\n";
            return 1;
        }
        write_all(argv[3], scores);
    } catch (const std::exception& e) {
        std::cerr << "unexpected exception: " << e.what() << "\n";
        return 1;
    }
    // the reference's error behaviour: rejected arguments throw invalid_argument
    try {
        const std::vector<ParamLimit> bad{{5.0, 1.0}};
        const search::PulsarSearchConfig cfg(1000, tsamp, nbins, eta, bad);  // nsamps not a power of two
        std::cerr << "expected std::invalid_argument\n";
        return 1;
    } catch (const std::invalid_argument&) {
    }
    try {
        // use_fourier defaults to true, as the reference's
        const search::PulsarSearchConfig cfg(nsamps, tsamp, nbins, eta, limits, 0.2, 1.5, true, 1, std::nullopt,
                                             std::nullopt, 5.0, widths);
        algorithms::FFACUDA<ComplexTypeCUDA> ffa(cfg);
        const auto& plan = ffa.get_plan();
        std::vector<ComplexType> cfold(plan.get_fold_size());
        ffa.execute(ts_e, ts_v, cfold);
        // the overload pair: a float span receives the fold back in time
        std::vector<float> tfold(plan.get_buffer_size_time());
        ffa.execute(ts_e, ts_v, tfold);
        if (plan.get_fold_size_time() != plan.get_fold_size() / plan_nbins_f(nbins) * nbins) {
            std::cerr << "fold_size_time mismatch\n";
            return 1;
        }
        write_all(argv[4], cfold);
        auto [scores, tplan] = algorithms::compute_ffa_scores_cuda(ts_e, ts_v, cfg);
        write_all(argv[5], scores);
    } catch (const std::exception& e) {
        std::cerr << "unexpected exception (Fourier path): " << e.what() << "\n";
        return 1;
    }
    std::cout << "ffacuda_check: ok\n";
    return 0;
}
