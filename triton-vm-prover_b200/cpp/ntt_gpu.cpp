// triton_vm::NTT and triton_vm::LDE (include/ntt/ntt.hpp) on the GPU, in place
// of the reference's src/ntt/ntt.cpp.  Same results, same exceptions:
// std::invalid_argument for a length that is not a power of two
// (src/ntt/ntt.cpp:59-86).
#include <algorithm>

#include "ntt/ntt.hpp"
#include "shim.hpp"

namespace triton_vm {

using tvmc_shim::check;
using tvmc_shim::words;

// NTT::forward (src/ntt/ntt.cpp:59-71): natural order in and out, w = 7^((p-1)/n).
void NTT::forward(std::vector<BFieldElement>& coeffs) {
    if (coeffs.empty()) throw std::invalid_argument("NTT size must be a power of 2");
    check(tvmc_ntt_host(words(coeffs.data()), coeffs.size(), 1, 0));
}

// NTT::inverse (src/ntt/ntt.cpp:73-86): w^-1 and the 1/n scale.
void NTT::inverse(std::vector<BFieldElement>& evals) {
    if (evals.empty()) throw std::invalid_argument("NTT size must be a power of 2");
    check(tvmc_ntt_host(words(evals.data()), evals.size(), 1, 1));
}

std::vector<BFieldElement> NTT::interpolate(const std::vector<BFieldElement>& column) {
    std::vector<BFieldElement> coeffs = column;
    inverse(coeffs);
    return coeffs;
}

// NTT::evaluate_on_coset (src/ntt/ntt.cpp:94-117): coefficients beyond
// domain_length are dropped, as in the reference.
std::vector<BFieldElement> NTT::evaluate_on_coset(const std::vector<BFieldElement>& coeffs, size_t domain_length,
                                                  BFieldElement offset) {
    if (domain_length == 0) throw std::invalid_argument("NTT size must be a power of 2");
    std::vector<BFieldElement> out(domain_length);
    check(tvmc_evaluate_on_coset_host(coeffs.empty() ? nullptr : words(coeffs.data()), coeffs.size(), 1,
                                      words(out.data()), domain_length, offset.value()));
    return out;
}

// LDE::extend_column (src/ntt/ntt.cpp:121-131): the trace domain's offset is
// not used, as in the reference.  Shapes outside the fused kernels' range go
// through the GPU interpolate + evaluate_on_coset pair.
std::vector<BFieldElement> LDE::extend_column(const std::vector<BFieldElement>& trace_column,
                                              const ArithmeticDomain& trace_domain,
                                              const ArithmeticDomain& quotient_domain) {
    (void)trace_domain;
    const size_t n = trace_column.size(), L = quotient_domain.length;
    if (tvmc_shim::lde_shape_supported(n, L)) {
        std::vector<BFieldElement> out(L);
        check(tvmc_lde_host(words(trace_column.data()), 1, n, words(out.data()), L, quotient_domain.offset.value()));
        return out;
    }
    return NTT::evaluate_on_coset(NTT::interpolate(trace_column), L, quotient_domain.offset);
}

// LDE::extend_table (src/ntt/ntt.cpp:133-172): every column in one batched call.
std::vector<std::vector<BFieldElement>> LDE::extend_table(const std::vector<std::vector<BFieldElement>>& trace_table,
                                                          const ArithmeticDomain& trace_domain,
                                                          const ArithmeticDomain& quotient_domain) {
    (void)trace_domain;
    if (trace_table.empty()) return {};
    size_t n, w;
    std::vector<uint64_t> cm = tvmc_shim::to_column_major(trace_table, &n, &w);
    const size_t L = quotient_domain.length;
    std::vector<uint64_t> out(L * w);
    if (w) {
        if (tvmc_shim::lde_shape_supported(n, L)) {
            check(tvmc_lde_host(cm.data(), w, n, out.data(), L, quotient_domain.offset.value()));
        } else {
            if (L == 0) throw std::invalid_argument("NTT size must be a power of 2");
            check(tvmc_ntt_host(cm.data(), n, w, 1));
            check(tvmc_evaluate_on_coset_host(cm.data(), n, w, out.data(), L, quotient_domain.offset.value()));
        }
    }
    return tvmc_shim::to_rows(out.data(), L, w);
}

}  // namespace triton_vm
