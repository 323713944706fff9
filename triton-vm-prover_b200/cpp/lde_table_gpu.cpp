// triton_vm::LDETable (include/lde/lde_table.hpp) on the GPU, in place of the
// reference's src/lde/lde_table.cpp.  compute_lde_and_merkle runs the whole
// randomized commitment (LDE -> row hash -> tree) in one library call and
// never brings the LDE back to the host.
#include <algorithm>

#include "lde/lde_table.hpp"
#include "merkle/merkle_tree.hpp"
#include "shim.hpp"

namespace triton_vm {

using tvmc_shim::check;
using tvmc_shim::words;

namespace {
// Randomizer coefficients of every column, zero-padded to the longest (zero
// coefficients leave the polynomial unchanged): r[col*R + k].
std::vector<uint64_t> pack_randomizers(const std::vector<std::vector<BFieldElement>>& rnd, size_t* R) {
    *R = 0;
    for (const auto& r : rnd) *R = std::max(*R, r.size());
    std::vector<uint64_t> out(rnd.size() * *R, 0);
    for (size_t c = 0; c < rnd.size(); c++)
        for (size_t k = 0; k < rnd[c].size(); k++) out[c * *R + k] = rnd[c][k].value();
    return out;
}

void check_randomizer_count(const std::vector<std::vector<BFieldElement>>& rnd, size_t cols) {
    if (rnd.size() != cols) throw std::invalid_argument("Randomizer coefficients count must match column count");
}
}  // namespace

// LDETable::extend_table_with_randomizers (src/lde/lde_table.cpp:8-57): per
// column RandomizedLDE::extend_column_with_randomizer, all columns in one call.
std::vector<std::vector<BFieldElement>> LDETable::extend_table_with_randomizers(
    const std::vector<std::vector<BFieldElement>>& trace_table, const ArithmeticDomain& trace_domain,
    const ArithmeticDomain& quotient_domain, const std::vector<std::vector<BFieldElement>>& randomizer_coeffs) {
    if (trace_table.empty()) return {};
    size_t n, w;
    std::vector<uint64_t> cm = tvmc_shim::to_column_major(trace_table, &n, &w);
    check_randomizer_count(randomizer_coeffs, w);
    size_t R;
    std::vector<uint64_t> r = pack_randomizers(randomizer_coeffs, &R);
    const size_t L = quotient_domain.length;
    std::vector<uint64_t> out(L * w);
    if (w) tvmc_shim::check_trace_offset(n, trace_domain.offset);
    if (w)
        check(tvmc_lde_randomized_host(cm.data(), w, n, R ? r.data() : nullptr, R, out.data(), L,
                                       trace_domain.offset.value(), quotient_domain.offset.value(), 0));
    return tvmc_shim::to_rows(out.data(), L, w);
}

// LDETable::compute_merkle_tree (src/lde/lde_table.cpp:59-86): Tip5 hash_varlen
// of every row, then the Merkle tree.
std::pair<std::vector<Digest>, Digest> LDETable::compute_merkle_tree(
    const std::vector<std::vector<BFieldElement>>& lde_table) {
    if (lde_table.empty()) return {{}, Digest()};
    const size_t rows = lde_table.size(), width = lde_table[0].size();
    std::vector<Digest> digests(rows);
    bool uniform = true;
    for (const auto& row : lde_table) uniform = uniform && row.size() == width;
    if (uniform) {
        std::vector<uint64_t> rm(rows * width);
        for (size_t i = 0; i < rows; i++)
            std::copy(tvmc_shim::words(lde_table[i].data()), tvmc_shim::words(lde_table[i].data()) + width,
                      rm.begin() + i * width);
        uint64_t none = 0;
        check(tvmc_hash_varlen_host(rm.empty() ? &none : rm.data(), rows, width, words(digests.data())));
    } else {
        for (size_t i = 0; i < rows; i++) digests[i] = Tip5::hash_varlen(lde_table[i]);
    }
    MerkleTree tree(digests);
    return {digests, tree.root()};
}

// LDETable::compute_lde_and_merkle (src/lde/lde_table.cpp:88-101): the fused
// randomized commitment of the row-major table; only the root comes back.
Digest LDETable::compute_lde_and_merkle(const std::vector<std::vector<BFieldElement>>& trace_table,
                                       const ArithmeticDomain& trace_domain,
                                       const ArithmeticDomain& quotient_domain,
                                       const std::vector<std::vector<BFieldElement>>& randomizer_coeffs) {
    if (trace_table.empty()) return Digest();
    const size_t n = trace_table.size(), w = trace_table[0].size(), L = quotient_domain.length;
    check_randomizer_count(randomizer_coeffs, w);
    if (!tvmc_shim::lde_shape_supported(n, L) || w == 0) {
        // shapes the fused path does not take: the two steps, as the reference composes them
        return compute_merkle_tree(
                   extend_table_with_randomizers(trace_table, trace_domain, quotient_domain, randomizer_coeffs))
            .second;
    }
    std::vector<uint64_t> rm(n * w);
    for (size_t i = 0; i < n; i++) {
        if (trace_table[i].size() != w) throw std::invalid_argument("table rows differ in width");
        std::copy(words(trace_table[i].data()), words(trace_table[i].data()) + w, rm.begin() + i * w);
    }
    tvmc_shim::check_trace_offset(n, trace_domain.offset);
    size_t R;
    std::vector<uint64_t> r = pack_randomizers(randomizer_coeffs, &R);
    tvmc_commitment* c = nullptr;
    check(tvmc_commit_randomized(rm.data(), n, w, (uint32_t)(L / n), trace_domain.offset.value(),
                                 quotient_domain.offset.value(), R ? r.data() : nullptr, R,
                                 TVMC_TRACE_ROW_MAJOR | TVMC_DISCARD_LDE | TVMC_SYNC, nullptr, &c));
    Digest root;
    const int rc = tvmc_commitment_root(c, words(&root));
    tvmc_commitment_free(c);
    check(rc);
    return root;
}

}  // namespace triton_vm
