// Python module `lucaslehmer`: the reference's module surface (lucaslehmer.cpp:344-387), every
// Lucas-Lehmer entry point running on the B200 engine through the C-ABI (include/llgpu.h).
//
// Name-for-name with the reference so its driver (PerfNumMultiCLL.py) and tests run unchanged:
//   lucas_lehmer / _res / gmp_res64_after      exact engine (reference: GMP, lucaslehmer.cpp:29-58)
//   lucas_lehmer_split / _split_res            same exact engine; `depth` (the reference's CPU
//                                              thread split, lucaslehmer.cpp:147-179) is accepted
//                                              and has no effect on one GPU
//   lucas_lehmer_fft / _fft_res / fft_res64_after / fft_info
//                                              FP64 IBDWT engine (lucaslehmer.cpp:209-342)
//   set_fft_bits_per_word, fft_backend, bench_square, primes, mersenne_digits, mersenne_str,
//   gmp_version, class LucasLehmer             as in the reference
// The exact engine is the Goldilocks NTT where it has a length for p, else the FP64 engine,
// whose results are exact too (round-off guard at 0.4, redone at a longer length).
// Errors (no GPU, CUDA failure, unsupported p) raise RuntimeError. The GIL is released around
// every GPU call, so a ThreadPool of callers runs concurrently (lucaslehmer.cpp:38).
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/llgpu.h"

namespace py = pybind11;

namespace {

// res64 of the last test run on this thread (the reference keeps the same thread-local side
// channel, lucaslehmer.cpp:23)
thread_local unsigned long long t_last_res64 = 0;

[[noreturn]] void raise(int rc) {
    std::string msg = std::string("llgpu: ") + llg_status_string(rc);
    const char* d = llg_last_error();
    if (d && *d) msg += std::string(": ") + d;
    throw std::runtime_error(msg);
}

llg_result run(unsigned long p, unsigned long iters, int engine) {
    llg_result r{};
    int rc;
    {
        py::gil_scoped_release release;
        rc = llg_run(p, iters, engine, 0, &r, nullptr, 0);
    }
    if (rc != LLG_OK) raise(rc);
    t_last_res64 = r.res64;
    return r;
}

int exact_engine(unsigned long p) {
    return llg_ntt_length(p) ? LLG_ENGINE_NTT : LLG_ENGINE_FP64;
}

bool ll_exact(unsigned long p) {
    if (p < 3 || p % 2 == 0) {
        t_last_res64 = 0;
        return p == 2;
    }
    return run(p, 0, exact_engine(p)).is_zero != 0;
}

bool ll_fft(unsigned long p) {
    if (p < 3 || p % 2 == 0) {
        t_last_res64 = 0;
        return p == 2;
    }
    return run(p, 0, LLG_ENGINE_FP64).is_zero != 0;
}

std::vector<unsigned long> primes_in_range(unsigned long lo, unsigned long hi) {
    std::vector<unsigned long> out;
    if (hi < 2) return out;
    std::vector<bool> comp(hi + 1, false);
    for (unsigned long i = 2; i * i <= hi; ++i)
        if (!comp[i])
            for (unsigned long j = i * i; j <= hi; j += i) comp[j] = true;
    for (unsigned long i = (lo < 2 ? 2 : lo); i <= hi; ++i)
        if (!comp[i]) out.push_back(i);
    return out;
}

// Decimal string of 2^p - 1: binary -> base 10^18 by repeated doubling in 60-bit steps.
std::string mersenne_str(unsigned long p) {
    if (p == 0) return "0";
    const uint64_t BASE = 1000000000000000000ull;  // 10^18
    std::vector<uint64_t> d(1, 1);                 // little-endian base-10^18 digits of 2^p
    unsigned long left = p;
    while (left) {
        const unsigned s = left >= 59 ? 59u : (unsigned)left;
        left -= s;
        unsigned __int128 carry = 0;
        for (auto& x : d) {
            unsigned __int128 v = ((unsigned __int128)x << s) + carry;
            x = (uint64_t)(v % BASE);
            carry = v / BASE;
        }
        while (carry) {
            d.push_back((uint64_t)(carry % BASE));
            carry /= BASE;
        }
    }
    // subtract 1 (2^p ends in 2, 4, 6 or 8, so no borrow)
    d[0] -= 1;
    std::string out = std::to_string(d.back());
    char buf[32];
    for (size_t i = d.size() - 1; i-- > 0;) {
        std::snprintf(buf, sizeof buf, "%018llu", (unsigned long long)d[i]);
        out += buf;
    }
    return out;
}

size_t mersenne_digits(unsigned long p) {
    if (p < 4000) return mersenne_str(p).size();
    // 2^p - 1 has the digit count of 2^p (no power of two is a power of ten): floor(p log10 2) + 1.
    // p log10(2) is never within 1e-9 of an integer for the exponents this is used on; the
    // long-double product is good to ~1e-19 relative.
    const long double l = (long double)p * 0.30102999566398119521373889472449302677L;
    return (size_t)floorl(l) + 1;
}

double bench_square(unsigned long bits, int iters, int depth) {
    (void)depth;
    unsigned long p = bits | 1ul;
    if (p < 3) p = 3;
    if (iters < 1) iters = 1;
    llg_result r = run(p, (unsigned long)iters, LLG_ENGINE_FP64);
    return r.seconds / (double)(r.iters ? r.iters : 1);
}

struct LucasLehmerCompat {};

}  // namespace

PYBIND11_MODULE(lucaslehmer, m, py::mod_gil_not_used()) {
    m.doc() = "Lucas-Lehmer Mersenne prime test on a B200 GPU (IBDWT FP64 + Goldilocks NTT engines)";
    m.def("lucas_lehmer", &ll_exact, py::arg("p"),
          "True iff 2^p - 1 is prime (Lucas-Lehmer), exact GPU engine. p should be prime.");
    m.def("lucas_lehmer_split", [](unsigned long p, int) { return ll_exact(p); }, py::arg("p"),
          py::arg("depth") = 1, "Same exact GPU engine; depth is accepted for compatibility.");
    m.def("lucas_lehmer_fft", &ll_fft, py::arg("p"),
          "Lucas-Lehmer on the FP64 IBDWT GPU engine (exact: longer transform on round-off trouble).");
    m.def("lucas_lehmer_res", [](unsigned long p) {
              bool r = ll_exact(p);
              return std::make_pair(r, t_last_res64);
          },
          py::arg("p"), "(is_prime, res64) on the exact engine: res64 = low 64 bits of the final residue.");
    m.def("lucas_lehmer_split_res", [](unsigned long p, int) {
              bool r = ll_exact(p);
              return std::make_pair(r, t_last_res64);
          },
          py::arg("p"), py::arg("depth") = 1, "(is_prime, res64), exact engine.");
    m.def("lucas_lehmer_fft_res", [](unsigned long p) {
              bool r = ll_fft(p);
              return std::make_pair(r, t_last_res64);
          },
          py::arg("p"), "(is_prime, res64) on the FP64 IBDWT engine (exact).");
    m.def("fft_res64_after", [](unsigned long p, unsigned long iters) {
              if (p < 3 || p % 2 == 0) return std::make_pair(0ull, 0.0);
              llg_result r = run(p, iters ? iters : p, LLG_ENGINE_FP64);
              return std::make_pair((unsigned long long)r.res64, r.max_err);
          },
          py::arg("p"), py::arg("iters"),
          "(res64, worst rounding error) after only `iters` squarings, FP64 engine.");
    m.def("gmp_res64_after", [](unsigned long p, unsigned long iters) {
              if (p < 3 || p % 2 == 0) return 0ull;
              return (unsigned long long)run(p, iters ? iters : p, exact_engine(p)).res64;
          },
          py::arg("p"), py::arg("iters"), "res64 after only `iters` squarings on the exact engine.");
    m.def("fft_info", [](unsigned long p) {
              size_t n = llg_fft_length(p, 0);
              double err = 0.0;
              if (p >= 3 && p % 2 == 1) {
                  llg_result r = run(p, 0, LLG_ENGINE_FP64);
                  err = r.max_err;
                  if (r.n) n = r.n;
              }
              return std::make_tuple(n, n ? (double)p / (double)n : 0.0, err);
          },
          py::arg("p"), "(FFT length, bits per word, worst rounding error) of an FP64-engine test of p.");
    m.attr("fft_backend") = std::string("b200-fp64-ibdwt");
    m.def("set_fft_bits_per_word", [](double b) {
              int rc = llg_set_max_bpw(b);
              if (rc) raise(rc);
          },
          py::arg("bits"), "Max bits per FFT word (default 18). Higher = shorter FFT, more round-off.");
    m.def("bench_square", &bench_square, py::arg("bits"), py::arg("iters") = 20, py::arg("depth") = 0,
          "device seconds per Lucas-Lehmer squaring at an exponent of `bits` bits (FP64 engine)");
    m.def("primes", &primes_in_range, py::arg("lo"), py::arg("hi"), "List of primes in [lo, hi].");
    m.def("mersenne_digits", &mersenne_digits, py::arg("p"), "Number of decimal digits of 2^p - 1.");
    m.def("mersenne_str", &mersenne_str, py::arg("p"), "Decimal string of 2^p - 1.");
    m.attr("gmp_version") = std::string("none (b200 engine)");
    py::class_<LucasLehmerCompat>(m, "LucasLehmer", py::module_local())
        .def(py::init<>())
        .def("sa_lucaslehmer", [](LucasLehmerCompat&, unsigned long p, py::object) { return ll_exact(p); },
             py::arg("N_"), py::arg("S_") = py::none())
        .def("sa_getListOfPrimes", [](LucasLehmerCompat&, py::list primes, unsigned long lo, unsigned long hi) {
            for (auto v : primes_in_range(lo, hi)) primes.append(v);
            return true;
        });
}
