// Python module `lucaslehmer_cuda`: the reference's GPU module surface (cuda/ll_ntt.cu:274-281)
// on the B200 engine, through the C-ABI (include/llgpu.h).
//
//   lucas_lehmer_batch(exponents, engine="fp64") -> [(p, is_prime, seconds, res64)]
//       every exponent in one call: grouped by transform length, one batched whole-test launch
//       per group. Results come back in input order (the reference's come back grouped by length;
//       callers index them by p). seconds < 0 marks an exponent the engine cannot take, as in the
//       reference (cuda/ll_ntt.cu:259-267). engine="ntt" selects the exact Goldilocks engine.
//   ntt_length(p)   transform length the batch engine groups p under (0 = cannot take; the
//                   driver routes those to its per-exponent path). Reference: ll_ntt.cu:176-180.
//   max_exponent()  largest p the batch engine takes. Reference: ll_ntt.cu:279.
//   device_info()   (name, SM count, global memory bytes). Reference: ll_ntt.cu:269-272.
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/llgpu.h"

namespace py = pybind11;

namespace {

[[noreturn]] void raise(int rc) {
    std::string msg = std::string("llgpu: ") + llg_status_string(rc);
    const char* d = llg_last_error();
    if (d && *d) msg += std::string(": ") + d;
    throw std::runtime_error(msg);
}

int engine_of(const std::string& e) {
    if (e == "fp64") return LLG_ENGINE_FP64;
    if (e == "ntt") return LLG_ENGINE_NTT;
    throw std::invalid_argument("engine must be 'fp64' or 'ntt'");
}

std::vector<std::tuple<unsigned long long, bool, double, unsigned long long>> batch(
    std::vector<unsigned long long> ps, const std::string& engine) {
    const int eng = engine_of(engine);
    std::vector<uint64_t> in(ps.begin(), ps.end());
    std::vector<llg_result> out(in.size());
    int rc;
    {
        py::gil_scoped_release release;
        rc = llg_run_batch(in.data(), in.size(), 0, eng, out.data(), nullptr, 0);
    }
    if (rc != LLG_OK) raise(rc);
    std::vector<std::tuple<unsigned long long, bool, double, unsigned long long>> res;
    res.reserve(in.size());
    for (size_t i = 0; i < in.size(); ++i) {
        const llg_result& r = out[i];
        if (r.status != LLG_OK)
            res.emplace_back(in[i], false, -1.0, 0ull);
        else
            res.emplace_back(in[i], r.is_zero != 0, r.seconds, (unsigned long long)r.res64);
    }
    return res;
}

unsigned long long batch_length(unsigned long long p) {
    uint32_t n = llg_ntt_length(p);
    if (!n) n = llg_fft_length(p, 0);
    return n;
}

}  // namespace

PYBIND11_MODULE(lucaslehmer_cuda, m, py::mod_gil_not_used()) {
    m.doc() = "Lucas-Lehmer on a B200: batched whole-test kernels, FP64 IBDWT and Goldilocks NTT";
    m.def("lucas_lehmer_batch", &batch, py::arg("exponents"), py::arg("engine") = std::string("fp64"),
          "[(p, is_prime, seconds, res64)] for a list of exponents; seconds < 0 marks one the "
          "engine cannot take.");
    m.def("ntt_length", &batch_length, py::arg("p"), "Transform length used for p (0 = cannot take).");
    m.def("max_exponent", []() {
              unsigned long long a = llg_max_exponent(LLG_ENGINE_FP64), b = llg_max_exponent(LLG_ENGINE_NTT);
              return a > b ? a : b;
          },
          "Largest p the batch engine handles.");
    m.def("device_info", []() {
        char name[256];
        int sms = 0;
        uint64_t mem = 0;
        int rc = llg_device_info(name, sizeof name, &sms, &mem);
        if (rc != LLG_OK) raise(rc);
        return std::make_tuple(std::string(name), sms, (size_t)mem);
    }, "(name, SM count, global memory bytes)");
}
