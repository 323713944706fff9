// The reference's own TableCommitment (src/table/table_commitment.cpp, compiled
// unchanged) running on the GPU through the C++ drop-in layer (TEST
// INFRASTRUCTURE).  Built by tests/cpp/Makefile with -ffunction-sections and
// --gc-sections, so TableCommitment::commit(const MasterMainTable&) -- the one
// function that needs the master table, which this check does not construct --
// is dropped at link time; every other function of the file is exercised.
//
// check (default): for main-like and aux-like tables, the caller-level path of
// MasterMainTable::low_degree_extend (src/table/master_table.cpp:2334-2372: per
// column LDE::extend_column, scattered into rows), then hash_bfield_row /
// hash_xfield_row per row, TableCommitment::from_digests, root,
// authentication_path, authentication_structure and TableCommitment::verify --
// compared with the CPU oracle.  Prints "table commitment check: N checks, F failed".
//
// time <log_n> <width>: times that per-column loop (the reference caller's own
// structure, one GPU round trip per column) against one batched drop-in call
// (LDE::extend_table) on the same table, and prints one JSON line.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lde/lde_table.hpp"
#include "merkle/merkle_tree.hpp"
#include "ntt/ntt.hpp"
#include "table/table_commitment.hpp"

extern "C" {
int tvmo_lde_column(const uint64_t* trace, size_t n, uint64_t* out, size_t L, uint64_t offset);
void tvmo_hash_varlen(const uint64_t* in, size_t n, uint64_t out[5]);
int tvmo_merkle_build(const uint64_t* leaves, size_t n, uint64_t* nodes);
long tvmo_auth_structure_indices(size_t n, const size_t* leaves, size_t m, size_t* out, size_t max_out);
uint64_t tvmo_primitive_root(uint32_t log2_order);
}

using namespace triton_vm;

namespace {
int g_checks = 0, g_failed = 0;
void expect(bool ok, const std::string& what) {
    g_checks++;
    if (!ok) {
        g_failed++;
        std::printf("FAIL %s\n", what.c_str());
    }
}
uint64_t g_rng = 0x7E5EED07;
uint64_t next_u64() {  // splitmix64
    uint64_t z = (g_rng += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
constexpr uint64_t P = 0xFFFFFFFF00000001ull;
ArithmeticDomain domain(size_t len, uint64_t offset) {
    ArithmeticDomain d;
    d.length = len;
    d.offset = BFieldElement(offset);
    uint32_t k = 0;
    while ((size_t(1) << k) < len) k++;
    d.generator = BFieldElement(tvmo_primitive_root(k));
    return d;
}
bool same(const Digest& d, const uint64_t* w) {
    for (size_t i = 0; i < 5; i++)
        if (d[i].value() != w[i]) return false;
    return true;
}

// The caller-level LDE of MasterMainTable::low_degree_extend: one column at a
// time through LDE::extend_column, written back row by row.
std::vector<std::vector<BFieldElement>> per_column_lde(const std::vector<std::vector<BFieldElement>>& rows,
                                                       size_t L) {
    const size_t n = rows.size(), w = rows[0].size();
    std::vector<std::vector<BFieldElement>> lde(L, std::vector<BFieldElement>(w));
    const ArithmeticDomain td = domain(n, 1), qd = domain(L, 7);
    std::vector<BFieldElement> col(n);
    for (size_t c = 0; c < w; c++) {
        for (size_t r = 0; r < n; r++) col[r] = rows[r][c];
        const std::vector<BFieldElement> e = LDE::extend_column(col, td, qd);
        for (size_t r = 0; r < L; r++) lde[r][c] = e[r];
    }
    return lde;
}

void check_table(size_t n, size_t w, bool xfe) {
    const size_t L = 4 * n;
    std::vector<std::vector<BFieldElement>> rows(n, std::vector<BFieldElement>(w));
    for (auto& r : rows)
        for (auto& x : r) x = BFieldElement(next_u64() % P);
    const auto lde = per_column_lde(rows, L);
    // oracle: the same LDE column by column, row digests, heap tree
    std::vector<uint64_t> col(n), ocol(L), olde(L * w);
    for (size_t c = 0; c < w; c++) {
        for (size_t r = 0; r < n; r++) col[r] = rows[r][c].value();
        tvmo_lde_column(col.data(), n, ocol.data(), L, 7);
        for (size_t r = 0; r < L; r++) olde[r * w + c] = ocol[r];
    }
    bool lde_ok = true;
    for (size_t r = 0; r < L && lde_ok; r++)
        for (size_t c = 0; c < w; c++)
            if (lde[r][c].value() != olde[r * w + c]) lde_ok = false;
    const std::string tag = std::string(xfe ? "aux " : "main ") + std::to_string(n) + "x" + std::to_string(w);
    expect(lde_ok, tag + " per-column LDE");
    std::vector<uint64_t> leaves(5 * L), nodes(10 * L);
    for (size_t r = 0; r < L; r++) tvmo_hash_varlen(olde.data() + r * w, w, leaves.data() + 5 * r);
    tvmo_merkle_build(leaves.data(), L, nodes.data());
    // the reference's row hashing and TableCommitment over the drop-in
    std::vector<Digest> digests(L);
    for (size_t r = 0; r < L; r++) {
        if (xfe) {  // the row as XFieldElements (c0, c1, c2) -- w is a multiple of 3
            std::vector<XFieldElement> xr(w / 3);
            for (size_t k = 0; k < w / 3; k++) xr[k] = XFieldElement(lde[r][3 * k], lde[r][3 * k + 1], lde[r][3 * k + 2]);
            digests[r] = hash_xfield_row(xr);
        } else {
            digests[r] = hash_bfield_row(lde[r]);
        }
    }
    bool dig_ok = true;
    for (size_t r = 0; r < L; r++) dig_ok = dig_ok && same(digests[r], leaves.data() + 5 * r);
    expect(dig_ok, tag + (xfe ? " hash_xfield_row" : " hash_bfield_row"));
    const TableCommitment tc = TableCommitment::from_digests(digests);
    expect(same(tc.root(), nodes.data() + 5), tag + " TableCommitment root");
    expect(tc.num_rows() == L, tag + " num_rows");
    for (size_t i : {size_t(0), size_t(1), L / 3, L - 1}) {
        const std::vector<Digest> path = tc.authentication_path(i);
        bool ok = path.size() == (size_t)__builtin_ctzll(L);
        size_t node = L + i;
        for (size_t k = 0; k < path.size() && ok; k++, node >>= 1) ok = same(path[k], nodes.data() + 5 * (node ^ 1));
        expect(ok, tag + " authentication_path " + std::to_string(i));
        expect(TableCommitment::verify(tc.root(), i, digests[i], path), tag + " verify " + std::to_string(i));
        // a leaf that differs in one element (another row's digest may equal this one:
        // the LDE of a one-row trace is constant)
        Digest wrong = digests[i];
        wrong[2] = wrong[2] + BFieldElement(1);
        expect(!TableCommitment::verify(tc.root(), i, wrong, path), tag + " verify rejects a wrong leaf " + std::to_string(i));
    }
    const std::vector<size_t> idx = {L - 1, 0, L / 2, 3 % L};
    const std::vector<Digest> st = tc.authentication_structure(idx);
    std::vector<size_t> exp_nodes(64 * idx.size());
    const long m = tvmo_auth_structure_indices(L, idx.data(), idx.size(), exp_nodes.data(), exp_nodes.size());
    bool ok = m >= 0 && st.size() == (size_t)m;
    for (long k = 0; k < m && ok; k++) ok = same(st[k], nodes.data() + 5 * exp_nodes[k]);
    expect(ok, tag + " authentication_structure");
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int time_lde(int log_n, size_t w) {
    const size_t n = size_t(1) << log_n, L = 4 * n;
    std::vector<std::vector<BFieldElement>> rows(n, std::vector<BFieldElement>(w));
    for (auto& r : rows)
        for (auto& x : r) x = BFieldElement(next_u64() % P);
    per_column_lde(rows, L);  // warm-up (tables, scratch)
    double t0 = now_s();
    const auto a = per_column_lde(rows, L);
    const double per_col = now_s() - t0;
    LDE::extend_table(rows, domain(n, 1), domain(L, 7));
    t0 = now_s();
    const auto b = LDE::extend_table(rows, domain(n, 1), domain(L, 7));
    const double batched = now_s() - t0;
    bool same_lde = a.size() == b.size();
    for (size_t r = 0; r < L && same_lde; r++) same_lde = a[r] == b[r];
    std::printf("{\"trace_len\": %zu, \"width\": %zu, \"per_column_extend_column_s\": %.4f, "
                "\"per_column_ms_per_column\": %.3f, \"extend_table_s\": %.4f, \"equal\": %s}\n",
                n, w, per_col, 1e3 * per_col / w, batched, same_lde ? "true" : "false");
    return same_lde ? 0 : 1;
}
}  // namespace

int main(int argc, char** argv) {
    if (argc == 4 && !std::strcmp(argv[1], "time")) return time_lde(std::atoi(argv[2]), (size_t)std::atoll(argv[3]));
    check_table(1, 7, false);
    check_table(64, 379, false);
    check_table(256, 23, false);
    check_table(128, 264, true);
    check_table(1024, 30, true);
    std::printf("table commitment check: %d checks, %d failed\n", g_checks, g_failed);
    return g_failed ? 1 : 0;
}
