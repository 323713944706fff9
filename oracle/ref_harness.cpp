// Harness over the reference prover's OWN C++ sources (TEST INFRASTRUCTURE ONLY).
//
// Built by oracle/Makefile into oracle/_ref/libtvm_ref.so from the unchanged
// reference files src/ntt/ntt.cpp, src/types/{b_field_element,x_field_element,digest}.cpp,
// src/hash/tip5.cpp, src/merkle/merkle_tree.cpp and src/lde/{lde_randomized,lde_table}.cpp.  It exposes a C ABI so
// that Python tests can (1) pin the C restatement in tvm_oracle.c against the
// reference itself and (2) time the reference's CPU path as the benchmark's
// CPU baseline.  The OpenMP loops over columns and rows are this harness's
// own; the per-column and per-row work is the reference's functions
// (LDE::extend_column, Tip5::hash_varlen, MerkleTree), called as the
// reference's MasterMainTable::low_degree_extend (src/table/master_table.cpp:2334-2372)
// and Stark::prove_with_table (src/stark.cpp:1163-1196) call them.
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "hash/tip5.hpp"
#include "lde/lde_randomized.hpp"
#include "lde/lde_table.hpp"
#include "merkle/merkle_tree.hpp"
#include "ntt/ntt.hpp"
#include "types/b_field_element.hpp"
#include "types/digest.hpp"

using namespace triton_vm;

namespace {
ArithmeticDomain domain(size_t len, uint64_t offset) {
    ArithmeticDomain d;
    d.length = len;
    d.offset = BFieldElement(offset);
    uint32_t k = 0;
    while ((size_t(1) << k) < len) k++;
    d.generator = BFieldElement::primitive_root_of_unity(k);
    return d;
}
void put_digest(const Digest& d, uint64_t* out) {
    for (size_t i = 0; i < Digest::LEN; i++) out[i] = d[i].value();
}
Digest get_digest(const uint64_t* in) {
    return Digest(BFieldElement(in[0]), BFieldElement(in[1]), BFieldElement(in[2]),
                  BFieldElement(in[3]), BFieldElement(in[4]));
}
}  // namespace

extern "C" {

int tvmr_max_threads() { return omp_get_max_threads(); }

void tvmr_set_threads(int n) { omp_set_num_threads(n); }

uint64_t tvmr_primitive_root(uint32_t k) { return BFieldElement::primitive_root_of_unity(k).value(); }

void tvmr_tip5_permutation(uint64_t* st) {
    Tip5 t;
    for (size_t i = 0; i < Tip5::STATE_SIZE; i++) t.state[i] = BFieldElement(st[i]);
    t.permutation();
    for (size_t i = 0; i < Tip5::STATE_SIZE; i++) st[i] = t.state[i].value();
}

void tvmr_hash_varlen(const uint64_t* in, size_t n, uint64_t* out) {
    std::vector<BFieldElement> v(n);
    for (size_t i = 0; i < n; i++) v[i] = BFieldElement(in[i]);
    put_digest(Tip5::hash_varlen(v), out);
}

void tvmr_hash_pair(const uint64_t* l, const uint64_t* r, uint64_t* out) {
    put_digest(Tip5::hash_pair(get_digest(l), get_digest(r)), out);
}

void tvmr_ntt(uint64_t* a, size_t n, int inverse) {
    std::vector<BFieldElement> v(n);
    for (size_t i = 0; i < n; i++) v[i] = BFieldElement(a[i]);
    if (inverse) NTT::inverse(v); else NTT::forward(v);
    for (size_t i = 0; i < n; i++) a[i] = v[i].value();
}

// NTT::evaluate_on_coset (src/ntt/ntt.cpp:94-117) of one coefficient vector.
void tvmr_evaluate_on_coset(const uint64_t* coeffs, size_t n, uint64_t* out, size_t L, uint64_t offset) {
    std::vector<BFieldElement> c(n);
    for (size_t i = 0; i < n; i++) c[i] = BFieldElement(coeffs[i]);
    std::vector<BFieldElement> e = NTT::evaluate_on_coset(c, L, BFieldElement(offset));
    for (size_t j = 0; j < L; j++) out[j] = e[j].value();
}

// Column-major LDE of `width` columns: trace[c*n + r] -> lde[c*L + r].
void tvmr_lde_table(const uint64_t* trace, size_t n, size_t width, uint64_t* lde, size_t L,
                    uint64_t offset) {
    ArithmeticDomain td = domain(n, 1), qd = domain(L, offset);
#pragma omp parallel for schedule(dynamic, 1)
    for (long c = 0; c < (long)width; c++) {
        std::vector<BFieldElement> col(n);
        for (size_t r = 0; r < n; r++) col[r] = BFieldElement(trace[c * n + r]);
        std::vector<BFieldElement> ext = LDE::extend_column(col, td, qd);
        for (size_t r = 0; r < L; r++) lde[c * L + r] = ext[r].value();
    }
}

// Leaf digests of rows [r0, r1) of a column-major table with `rows` rows.
void tvmr_hash_rows(const uint64_t* lde, size_t rows, size_t width, size_t r0, size_t r1,
                    uint64_t* digests) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long r = (long)r0; r < (long)r1; r++) {
        std::vector<BFieldElement> row(width);
        for (size_t c = 0; c < width; c++) row[c] = BFieldElement(lde[c * rows + r]);
        put_digest(Tip5::hash_varlen(row), digests + 5 * (r - r0));
    }
}

// Heap tree over n leaves: nodes[5*i .. 5*i+4] for i in [1, 2n); node 0 zeroed.
int tvmr_merkle(const uint64_t* leaves, size_t n, uint64_t* nodes) {
    std::vector<Digest> lv(n);
    for (size_t i = 0; i < n; i++) lv[i] = get_digest(leaves + 5 * i);
    try {
        MerkleTree t(lv);
        std::memset(nodes, 0, 40);
        put_digest(t.root(), nodes + 5);
        // Every node is reachable as an authentication-path entry or a leaf;
        // walk all leaves' paths to recover the full heap.
        for (size_t i = 0; i < n; i++) put_digest(t.leaf(i), nodes + 5 * (n + i));
        for (size_t i = 0; i < n; i += 2) {
            std::vector<Digest> p = t.authentication_path(i);
            size_t node = n + i;
            for (size_t k = 0; k < p.size(); k++, node >>= 1) put_digest(p[k], nodes + 5 * (node ^ 1));
        }
    } catch (...) {
        return -1;
    }
    return 0;
}

int tvmr_auth_path(const uint64_t* leaves, size_t n, size_t leaf, uint64_t* out) {
    std::vector<Digest> lv(n);
    for (size_t i = 0; i < n; i++) lv[i] = get_digest(leaves + 5 * i);
    try {
        MerkleTree t(lv);
        std::vector<Digest> p = t.authentication_path(leaf);
        for (size_t k = 0; k < p.size(); k++) put_digest(p[k], out + 5 * k);
        return (int)p.size();
    } catch (...) {
        return -1;
    }
}

long tvmr_auth_structure(const uint64_t* leaves, size_t n, const size_t* idx, size_t m,
                         uint64_t* out, size_t max_out) {
    std::vector<Digest> lv(n);
    for (size_t i = 0; i < n; i++) lv[i] = get_digest(leaves + 5 * i);
    try {
        MerkleTree t(lv);
        std::vector<size_t> ix(idx, idx + m);
        std::vector<Digest> s = t.authentication_structure(ix);
        for (size_t k = 0; k < s.size() && k < max_out; k++) put_digest(s[k], out + 5 * k);
        return (long)s.size();
    } catch (...) {
        return -1;
    }
}

// The whole CPU commit of one table with the reference's functions:
// LDE per column, hash_varlen per row, MerkleTree over the leaves.
// Writes the root (5 words). Returns 0 on success.
int tvmr_commit(const uint64_t* trace, size_t n, size_t width, size_t L, uint64_t offset,
                uint64_t* lde, uint64_t* root) {
    tvmr_lde_table(trace, n, width, lde, L, offset);
    std::vector<uint64_t> d(5 * L);
    tvmr_hash_rows(lde, L, width, 0, L, d.data());
    std::vector<Digest> lv(L);
    for (size_t i = 0; i < L; i++) lv[i] = get_digest(d.data() + 5 * i);
    try {
        MerkleTree t(lv);
        put_digest(t.root(), root);
    } catch (...) {
        return -1;
    }
    return 0;
}

// RandomizedLDE::extend_column_with_randomizer (src/lde/lde_randomized.cpp:71-154)
// on each column-major column: trace[c*n + i] -> out[c*L + j]; randomizer
// coefficients rnd[c*R + k].
void tvmr_lde_randomized(const uint64_t* trace, size_t n, size_t width, const uint64_t* rnd, size_t R,
                         uint64_t* out, size_t L, uint64_t trace_offset, uint64_t offset) {
    const ArithmeticDomain td = domain(n, trace_offset), qd = domain(L, offset);
#pragma omp parallel for schedule(dynamic)
    for (long c = 0; c < (long)width; c++) {
        std::vector<BFieldElement> col(n), r(R);
        for (size_t i = 0; i < n; i++) col[i] = BFieldElement(trace[c * n + i]);
        for (size_t k = 0; k < R; k++) r[k] = BFieldElement(rnd[c * R + k]);
        auto e = RandomizedLDE::extend_column_with_randomizer(col, td, qd, r);
        for (size_t j = 0; j < L; j++) out[c * L + j] = e[j].value();
    }
}

// RandomizedLDE::extend_xfield_column_with_randomizer (xfe_rnd = 0, base-field
// randomizer rnd[c*R + k]) and extend_xfield_column_with_xfield_randomizer
// (xfe_rnd = 1, rnd[(c*R + k)*3 + limb]) on XFE columns trace[(c*n + i)*3 + limb];
// out[(c*L + j)*3 + limb].
void tvmr_lde_randomized_xfe(const uint64_t* trace, size_t n, size_t width, const uint64_t* rnd, size_t R,
                             int xfe_rnd, uint64_t* out, size_t L, uint64_t trace_offset, uint64_t offset) {
    const ArithmeticDomain td = domain(n, trace_offset), qd = domain(L, offset);
    auto xfe = [](const uint64_t* v) {
        return XFieldElement(BFieldElement(v[0]), BFieldElement(v[1]), BFieldElement(v[2]));
    };
#pragma omp parallel for schedule(dynamic)
    for (long c = 0; c < (long)width; c++) {
        std::vector<XFieldElement> col(n);
        for (size_t i = 0; i < n; i++) col[i] = xfe(trace + 3 * (c * n + i));
        std::vector<XFieldElement> e;
        if (xfe_rnd) {
            std::vector<XFieldElement> r(R);
            for (size_t k = 0; k < R; k++) r[k] = xfe(rnd + 3 * (c * R + k));
            e = RandomizedLDE::extend_xfield_column_with_xfield_randomizer(col, td, qd, r);
        } else {
            std::vector<BFieldElement> r(R);
            for (size_t k = 0; k < R; k++) r[k] = BFieldElement(rnd[c * R + k]);
            e = RandomizedLDE::extend_xfield_column_with_randomizer(col, td, qd, r);
        }
        for (size_t j = 0; j < L; j++)
            for (int l = 0; l < 3; l++) out[3 * (c * L + j) + l] = e[j].coeff(l).value();
    }
}

// LDETable::compute_lde_and_merkle (src/lde/lde_table.cpp:88-101) on a
// row-major table rows[i*width + c] with randomizers rnd[c*R + k]; writes the
// root.  Returns 0, or -1 when the reference throws.
int tvmr_lde_table_root(const uint64_t* rows, size_t n, size_t width, const uint64_t* rnd, size_t R, size_t L,
                        uint64_t trace_offset, uint64_t offset, uint64_t* root) {
    std::vector<std::vector<BFieldElement>> t(n, std::vector<BFieldElement>(width));
    for (size_t i = 0; i < n; i++)
        for (size_t c = 0; c < width; c++) t[i][c] = BFieldElement(rows[i * width + c]);
    std::vector<std::vector<BFieldElement>> r(width, std::vector<BFieldElement>(R));
    for (size_t c = 0; c < width; c++)
        for (size_t k = 0; k < R; k++) r[c][k] = BFieldElement(rnd[c * R + k]);
    try {
        put_digest(LDETable::compute_lde_and_merkle(t, domain(n, trace_offset), domain(L, offset), r), root);
    } catch (...) {
        return -1;
    }
    return 0;
}

}  // extern "C"
