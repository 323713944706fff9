// triton_vm::RandomizedLDE (include/lde/lde_randomized.hpp) on the GPU, in
// place of the reference's src/lde/lde_randomized.cpp.  The zerofier helpers
// build the same small polynomials as the reference (x^n - offset^n and its
// product with a randomizer); the extensions run in the library's randomized
// LDE, which adds the zerofier-times-randomizer term inside the LDE kernels.
#include <algorithm>

#include "lde/lde_randomized.hpp"
#include "ntt/ntt.hpp"
#include "shim.hpp"

namespace triton_vm {

using tvmc_shim::check;
using tvmc_shim::words;

// x^n - offset^n (src/lde/lde_randomized.cpp:10-35).
BPolynomial RandomizedLDE::compute_zerofier(const ArithmeticDomain& domain) {
    if (domain.length == 0) throw std::invalid_argument("Domain length must be > 0");
    BPolynomial z = BPolynomial::x_to_the(domain.length);
    if (domain.offset.value() != 0) z[0] = BFieldElement(0) - domain.offset.pow(domain.length);
    return z;
}

// x^n p(x) - offset^n p(x) (src/lde/lde_randomized.cpp:37-68).
BPolynomial RandomizedLDE::mul_zerofier_with(const ArithmeticDomain& domain, const BPolynomial& polynomial) {
    const size_t n = domain.length, m = polynomial.size();
    const BFieldElement on = domain.offset.pow(n);
    std::vector<BFieldElement> c(n + m, BFieldElement(0));
    for (size_t i = 0; i < m; i++) c[n + i] = polynomial[i];
    for (size_t i = 0; i < m; i++) c[i] = c[i] - polynomial[i] * on;
    return BPolynomial(c);
}

// RandomizedLDE::extend_column_with_randomizer (src/lde/lde_randomized.cpp:71-154).
std::vector<BFieldElement> RandomizedLDE::extend_column_with_randomizer(
    const std::vector<BFieldElement>& trace_column, const ArithmeticDomain& trace_domain,
    const ArithmeticDomain& target_domain, const std::vector<BFieldElement>& randomizer_coeffs) {
    tvmc_shim::check_trace_offset(trace_column.size(), trace_domain.offset);
    const size_t L = target_domain.length;
    std::vector<BFieldElement> out(L);
    check(tvmc_lde_randomized_host(words(trace_column.data()), 1, trace_column.size(),
                                   randomizer_coeffs.empty() ? nullptr : words(randomizer_coeffs.data()),
                                   randomizer_coeffs.size(), words(out.data()), L, trace_domain.offset.value(),
                                   target_domain.offset.value(), 0));
    return out;
}

namespace {
// XFE columns as three limb columns; limb k of randomizer coefficient j is
// rnd(j, k).  The reference's XFE variants cut the polynomial at the target
// length (src/lde/lde_randomized.cpp:246-251): TVMC_RAND_TRUNCATE.
template <typename RndLimb>
std::vector<XFieldElement> extend_xfe(const std::vector<XFieldElement>& col, const ArithmeticDomain& td,
                                      const ArithmeticDomain& qd, size_t R, RndLimb rnd) {
    const size_t n = col.size(), L = qd.length;
    tvmc_shim::check_trace_offset(n, td.offset);
    std::vector<uint64_t> limbs(3 * n), r(3 * R), out(3 * L);
    for (size_t i = 0; i < n; i++)
        for (size_t k = 0; k < 3; k++) limbs[k * n + i] = col[i].coeff(k).value();
    for (size_t j = 0; j < R; j++)
        for (size_t k = 0; k < 3; k++) r[k * R + j] = rnd(j, k);
    check(tvmc_lde_randomized_host(limbs.data(), 3, n, R ? r.data() : nullptr, R, out.data(), L,
                                   td.offset.value(), qd.offset.value(), TVMC_RAND_TRUNCATE));
    std::vector<XFieldElement> res(L);
    for (size_t j = 0; j < L; j++)
        res[j] = XFieldElement(BFieldElement(out[j]), BFieldElement(out[L + j]), BFieldElement(out[2 * L + j]));
    return res;
}
}  // namespace

// Base-field randomizer, lifted to the XFE's first limb (src/lde/lde_randomized.cpp:178-277).
std::vector<XFieldElement> RandomizedLDE::extend_xfield_column_with_randomizer(
    const std::vector<XFieldElement>& trace_column, const ArithmeticDomain& trace_domain,
    const ArithmeticDomain& quotient_domain, const std::vector<BFieldElement>& randomizer_coeffs) {
    return extend_xfe(trace_column, trace_domain, quotient_domain, randomizer_coeffs.size(),
                      [&](size_t j, size_t k) { return k == 0 ? randomizer_coeffs[j].value() : uint64_t(0); });
}

std::vector<XFieldElement> RandomizedLDE::extend_xfield_column_with_xfield_randomizer(
    const std::vector<XFieldElement>& trace_column, const ArithmeticDomain& trace_domain,
    const ArithmeticDomain& quotient_domain, const std::vector<XFieldElement>& randomizer_coeffs) {
    return extend_xfe(trace_column, trace_domain, quotient_domain, randomizer_coeffs.size(),
                      [&](size_t j, size_t k) { return randomizer_coeffs[j].coeff(k).value(); });
}

// RandomizedLDE::verify_zerofier (src/lde/lde_randomized.cpp:156-176): the
// polynomial vanishes on the whole domain.  Its evaluations on the domain are
// computed on the GPU: the coefficients folded modulo x^n - offset^n (chunk k
// of n coefficients scaled by offset^(kn)), then one coset evaluation.
bool RandomizedLDE::verify_zerofier(const ArithmeticDomain& domain, const BPolynomial& zerofier) {
    const size_t n = domain.length;
    if (n == 0) return true;
    const std::vector<BFieldElement>& c = zerofier.raw_coefficients();
    std::vector<BFieldElement> folded(n, BFieldElement(0));
    const BFieldElement on = domain.offset.pow(n);
    BFieldElement s = BFieldElement::one();
    for (size_t k0 = 0; k0 < c.size(); k0 += n, s = s * on)
        for (size_t i = 0; i < n && k0 + i < c.size(); i++) folded[i] = folded[i] + c[k0 + i] * s;
    std::vector<BFieldElement> ev;
    if ((n & (n - 1)) == 0) {
        ev = NTT::evaluate_on_coset(folded, n, domain.offset);
    } else {  // not an NTT size: the domain as listed by its generator
        ev.resize(n);
        BFieldElement x = domain.offset;
        for (size_t j = 0; j < n; j++, x = x * domain.generator) ev[j] = zerofier.evaluate(x);
    }
    return std::all_of(ev.begin(), ev.end(), [](const BFieldElement& v) { return v.value() == 0; });
}

}  // namespace triton_vm
