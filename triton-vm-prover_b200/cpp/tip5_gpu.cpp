// triton_vm::Tip5 (include/hash/tip5.hpp) on the GPU, in place of the
// reference's src/hash/tip5.cpp.  The public parameter tables are filled from
// the library's own (tvmc_tip5_parameters), so they are the constants the
// kernels compute with.  Single-state calls (permutation, round, trace, the
// sponge) are one small GPU round trip each; row and pair hashing in bulk goes
// through MerkleTree, hash_row callers batching rows, or the C ABI directly.
#include <algorithm>

#include "hash/tip5.hpp"
#include "shim.hpp"

namespace triton_vm {

using tvmc_shim::check;
using tvmc_shim::words;

namespace {
struct Tip5Params {
    uint8_t lookup[256];
    uint64_t mds[16];
    uint64_t rc[80];
    Tip5Params() { tvmc_tip5_parameters(lookup, mds, rc); }
};
const Tip5Params& tip5_params() {
    static const Tip5Params p;
    return p;
}
}  // namespace

const std::array<uint8_t, 256> Tip5::LOOKUP_TABLE = [] {
    std::array<uint8_t, 256> a{};
    std::copy(tip5_params().lookup, tip5_params().lookup + 256, a.begin());
    return a;
}();

const std::array<int64_t, Tip5::STATE_SIZE> Tip5::MDS_MATRIX_FIRST_COLUMN = [] {
    std::array<int64_t, STATE_SIZE> a{};
    for (size_t i = 0; i < STATE_SIZE; i++) a[i] = (int64_t)tip5_params().mds[i];
    return a;
}();

const std::array<BFieldElement, Tip5::NUM_ROUNDS * Tip5::STATE_SIZE> Tip5::ROUND_CONSTANTS = [] {
    std::array<BFieldElement, NUM_ROUNDS * STATE_SIZE> a{};
    for (size_t i = 0; i < a.size(); i++) a[i] = BFieldElement(tip5_params().rc[i]);
    return a;
}();

Tip5::Tip5() { state.fill(BFieldElement::zero()); }

// Both sponge domains start from the all-zero state (src/hash/tip5.cpp:84-90).
Tip5 Tip5::init() { return Tip5(); }

void Tip5::permutation() { check(tvmc_tip5_permutation_batch_host(words(state.data()), 1)); }

void Tip5::round(size_t round_index) {
    if (round_index >= NUM_ROUNDS) throw std::invalid_argument("Tip5 round index out of range");
    check(tvmc_tip5_rounds_host(words(state.data()), 1, (uint32_t)round_index, 1, nullptr));
}

// Tip5::trace (src/hash/tip5.cpp:97-112): the state before and after each
// round; advances the state by one permutation.
std::vector<std::array<BFieldElement, Tip5::STATE_SIZE>> Tip5::trace() {
    std::vector<std::array<BFieldElement, STATE_SIZE>> t(NUM_ROUNDS + 1);
    t[0] = state;
    static_assert(sizeof(std::array<BFieldElement, STATE_SIZE>) == 8 * STATE_SIZE, "dense state rows");
    check(tvmc_tip5_rounds_host(words(state.data()), 1, 0, NUM_ROUNDS, words(t[1].data())));
    return t;
}

// Overwrite mode: at most RATE elements replace the rate, then one permutation
// (src/hash/tip5.cpp:205-211).
void Tip5::absorb(const std::vector<BFieldElement>& elements) {
    const size_t k = std::min(elements.size(), RATE);
    std::copy(elements.begin(), elements.begin() + k, state.begin());
    permutation();
}

std::vector<BFieldElement> Tip5::squeeze(size_t count) {
    return std::vector<BFieldElement>(state.begin(), state.begin() + std::min(count, RATE));
}

// Fixed-length domain: capacity ones, rate = input (src/hash/tip5.cpp:224-244);
// the library's pair hash is exactly this with input = left || right.
Digest Tip5::hash_10(const std::array<BFieldElement, RATE>& input) {
    Digest d;
    check(tvmc_hash_pairs_host(words(input.data()), words(input.data()) + 5, words(&d), 1));
    return d;
}

Digest Tip5::hash_varlen(const std::vector<BFieldElement>& input) {
    Digest d;
    uint64_t none = 0;
    check(tvmc_hash_varlen_host(input.empty() ? &none : words(input.data()), 1, input.size(), words(&d)));
    return d;
}

Digest Tip5::hash_pair(const Digest& left, const Digest& right) {
    Digest d;
    check(tvmc_hash_pairs_host(words(&left), words(&right), words(&d), 1));
    return d;
}

}  // namespace triton_vm
