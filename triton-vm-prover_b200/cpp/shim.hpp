// Shared helpers of the C++ drop-in layer.
//
// The files in this directory implement the reference prover's C++ classes
// for the commitment path -- NTT and LDE (include/ntt/ntt.hpp), LDETable
// (include/lde/lde_table.hpp), RandomizedLDE (include/lde/lde_randomized.hpp),
// Tip5 (include/hash/tip5.hpp), MerkleTree and hash_row
// (include/merkle/merkle_tree.hpp) -- on top of the tvmc C ABI (include/tvmc.h).
// They compile inside the reference's build, against its unchanged headers, in
// place of src/ntt/ntt.cpp, src/lde/lde_table.cpp, src/lde/lde_randomized.cpp,
// src/hash/tip5.cpp and src/merkle/merkle_tree.cpp, so that callers such as
// Stark::prove_with_table and MasterMainTable::low_degree_extend run on the GPU
// without a source change.  Every computation goes to the library; what stays
// here is argument checking, layout conversion and index bookkeeping.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "tvmc.h"
#include "types/b_field_element.hpp"
#include "types/digest.hpp"

namespace tvmc_shim {

using triton_vm::BFieldElement;
using triton_vm::Digest;

// The library exchanges plain u64 words; the reference's element types are
// exactly that in memory (one canonical u64; five of them).
static_assert(sizeof(BFieldElement) == 8 && alignof(BFieldElement) == 8, "BFieldElement is one u64");
static_assert(sizeof(Digest) == 40, "Digest is five BFieldElements");

// The reference reports bad sizes with std::invalid_argument and bad indices
// with std::out_of_range; the library's status codes map onto the same types.
[[noreturn]] inline void raise(int status) {
    const std::string msg = tvmc_last_error();
    switch (status) {
        case TVMC_ERR_INVALID:
        case TVMC_ERR_UNSUPPORTED: throw std::invalid_argument(msg);
        case TVMC_ERR_RANGE: throw std::out_of_range(msg);
        default: throw std::runtime_error(std::string("tvmc: ") + tvmc_status_string(status) + ": " + msg);
    }
}

inline void check(int status) {
    if (status != TVMC_OK) raise(status);
}

inline uint64_t* words(BFieldElement* p) { return reinterpret_cast<uint64_t*>(p); }
inline const uint64_t* words(const BFieldElement* p) { return reinterpret_cast<const uint64_t*>(p); }
inline uint64_t* words(Digest* p) { return reinterpret_cast<uint64_t*>(p); }
inline const uint64_t* words(const Digest* p) { return reinterpret_cast<const uint64_t*>(p); }

// Rows of a [rows][cols] table as column-major words; all rows must have the
// width of the first.
inline std::vector<uint64_t> to_column_major(const std::vector<std::vector<BFieldElement>>& t, size_t* rows,
                                             size_t* cols) {
    *rows = t.size();
    *cols = t.empty() ? 0 : t[0].size();
    std::vector<uint64_t> cm(*rows * *cols);
    for (size_t r = 0; r < *rows; r++) {
        if (t[r].size() != *cols) throw std::invalid_argument("table rows differ in width");
        for (size_t c = 0; c < *cols; c++) cm[c * *rows + r] = t[r][c].value();
    }
    return cm;
}

// Column-major words -> [rows][cols] table.
inline std::vector<std::vector<BFieldElement>> to_rows(const uint64_t* cm, size_t rows, size_t cols) {
    std::vector<std::vector<BFieldElement>> t(rows, std::vector<BFieldElement>(cols));
    for (size_t c = 0; c < cols; c++)
        for (size_t r = 0; r < rows; r++) t[r][c] = BFieldElement(cm[c * rows + r]);
    return t;
}

// The randomized LDE scales by the trace offset's inverse; the reference's
// BFieldElement::inverse raises std::domain_error for zero
// (src/types/b_field_element.cpp:139-146).  Checked after the length, as the
// reference's interpolation comes first.
inline void check_trace_offset(size_t trace_len, const BFieldElement& offset) {
    if (trace_len && !(trace_len & (trace_len - 1)) && offset.value() == 0)
        throw std::domain_error("Cannot invert zero");
}

// Shapes the fused LDE kernels take: a power-of-two trace of at most
// 2^TVMC_MAX_LOG_LDE_TRACE rows, extended by 2^k, 0 <= k <= 4.
inline bool lde_shape_supported(size_t trace_len, size_t target_len) {
    auto pow2 = [](size_t v) { return v && !(v & (v - 1)); };
    if (!pow2(trace_len) || !pow2(target_len) || target_len < trace_len) return false;
    if (trace_len > (size_t(1) << TVMC_MAX_LOG_LDE_TRACE)) return false;
    return target_len / trace_len <= 16;
}

}  // namespace tvmc_shim
