// Self-check of the C++ drop-in layer (TEST INFRASTRUCTURE).
//
// Calls every public function of the reference's NTT, LDE, LDETable,
// RandomizedLDE, Tip5 and MerkleTree classes and hash_row -- as implemented by
// triton-vm-prover_b200/cpp on the GPU -- through the reference's own headers,
// and compares each result with the CPU oracle (oracle/tvm_oracle.c) on the
// same seeded inputs, plus the exceptions the reference raises.  Prints one
// line per failed check and "shim selftest: N checks, F failed"; exits 0 only
// when every check passed.  Built by tests/cpp/Makefile.
#include <array>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "hash/tip5.hpp"
#include "lde/lde_randomized.hpp"
#include "lde/lde_table.hpp"
#include "merkle/merkle_tree.hpp"
#include "ntt/ntt.hpp"

extern "C" {
int tvmo_ntt_forward(uint64_t* a, size_t n);
int tvmo_ntt_inverse(uint64_t* a, size_t n);
int tvmo_evaluate_on_coset(const uint64_t* coeffs, size_t n, uint64_t* out, size_t L, uint64_t offset);
int tvmo_lde_column(const uint64_t* trace, size_t n, uint64_t* out, size_t L, uint64_t offset);
int tvmo_lde_randomized_column(const uint64_t* trace, size_t n, const uint64_t* r, size_t R, uint64_t* out,
                               size_t L, uint64_t t, uint64_t o, int truncate);
void tvmo_tip5_parameters(uint8_t lookup[256], uint64_t mds[16], uint64_t rc[80]);
void tvmo_tip5_permutation(uint64_t st[16]);
void tvmo_hash_varlen(const uint64_t* in, size_t n, uint64_t out[5]);
void tvmo_hash_10(const uint64_t in[10], uint64_t out[5]);
void tvmo_hash_pair(const uint64_t l[5], const uint64_t r[5], uint64_t out[5]);
int tvmo_merkle_build(const uint64_t* leaves, size_t n, uint64_t* nodes);
long tvmo_auth_structure_indices(size_t n, const size_t* leaves, size_t m, size_t* out, size_t max_out);
uint64_t tvmo_pow(uint64_t base, uint64_t e);
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

template <typename E>
void expect_throw(const std::function<void()>& f, const std::string& what) {
    bool got = false;
    try {
        f();
    } catch (const E&) {
        got = true;
    } catch (const std::exception& e) {
        std::printf("  (%s threw another exception: %s)\n", what.c_str(), e.what());
    }
    expect(got, what + " throws");
}

uint64_t g_rng = 0x7E5EED00;
uint64_t next_u64() {  // splitmix64
    uint64_t z = (g_rng += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
constexpr uint64_t P = 0xFFFFFFFF00000001ull;
BFieldElement rand_bfe() { return BFieldElement(next_u64() % P); }
std::vector<BFieldElement> rand_vec(size_t n) {
    std::vector<BFieldElement> v(n);
    for (auto& x : v) x = rand_bfe();
    return v;
}
std::vector<uint64_t> raw(const std::vector<BFieldElement>& v) {
    std::vector<uint64_t> r(v.size());
    for (size_t i = 0; i < v.size(); i++) r[i] = v[i].value();
    return r;
}
bool same(const std::vector<BFieldElement>& a, const std::vector<uint64_t>& b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); i++)
        if (a[i].value() != b[i]) return false;
    return true;
}
bool same(const Digest& d, const uint64_t* w) {
    for (size_t i = 0; i < 5; i++)
        if (d[i].value() != w[i]) return false;
    return true;
}
Digest digest_of(const uint64_t* w) {
    return Digest(BFieldElement(w[0]), BFieldElement(w[1]), BFieldElement(w[2]), BFieldElement(w[3]),
                  BFieldElement(w[4]));
}
ArithmeticDomain domain(size_t len, uint64_t offset) {
    ArithmeticDomain d;
    d.length = len;
    d.offset = BFieldElement(offset);
    uint32_t k = 0;
    while ((size_t(1) << k) < len) k++;
    d.generator = BFieldElement(tvmo_primitive_root(k));
    return d;
}
std::string S(const char* f, size_t a) { return std::string(f) + "(" + std::to_string(a) + ")"; }

void check_ntt() {
    for (size_t k = 0; k <= 14; k++) {
        const size_t n = size_t(1) << k;
        auto v = rand_vec(n);
        auto f = v, i = v;
        NTT::forward(f);
        NTT::inverse(i);
        auto rf = raw(v), ri = raw(v);
        tvmo_ntt_forward(rf.data(), n);
        tvmo_ntt_inverse(ri.data(), n);
        expect(same(f, rf), S("NTT::forward", n));
        expect(same(i, ri), S("NTT::inverse", n));
        expect(same(NTT::interpolate(v), ri), S("NTT::interpolate", n));
    }
    expect_throw<std::invalid_argument>([] { std::vector<BFieldElement> e; NTT::forward(e); }, "NTT::forward(0)");
    expect_throw<std::invalid_argument>([] { auto e = rand_vec(12); NTT::inverse(e); }, "NTT::inverse(12)");
    // evaluate_on_coset: shorter and longer coefficient vectors than the domain
    for (size_t nc : {5u, 16u, 40u}) {
        auto c = rand_vec(nc);
        auto got = NTT::evaluate_on_coset(c, 16, BFieldElement(7));
        std::vector<uint64_t> exp(16);
        tvmo_evaluate_on_coset(raw(c).data(), nc < 16 ? nc : 16, exp.data(), 16, 7);
        expect(same(got, exp), S("NTT::evaluate_on_coset", nc));
    }
    expect_throw<std::invalid_argument>([] { NTT::evaluate_on_coset(rand_vec(4), 0, BFieldElement(7)); },
                                        "NTT::evaluate_on_coset(L=0)");
}

void check_lde() {
    // the fused shapes, expansion above 16 and a target shorter than the trace
    for (auto [n, L] : std::vector<std::pair<size_t, size_t>>{{1, 4}, {64, 256}, {1024, 4096}, {16, 1024}, {64, 32}}) {
        auto col = rand_vec(n);
        auto got = LDE::extend_column(col, domain(n, 1), domain(L, 7));
        std::vector<uint64_t> exp(L), coeffs = raw(col);
        tvmo_ntt_inverse(coeffs.data(), n);
        tvmo_evaluate_on_coset(coeffs.data(), n < L ? n : L, exp.data(), L, 7);
        expect(same(got, exp), S("LDE::extend_column n", n) + S(" L", L));
    }
    const size_t n = 64, w = 7, L = 256;
    std::vector<std::vector<BFieldElement>> t(n);
    for (auto& r : t) r = rand_vec(w);
    auto lde = LDE::extend_table(t, domain(n, 1), domain(L, 7));
    bool ok = lde.size() == L;
    for (size_t c = 0; c < w && ok; c++) {
        std::vector<uint64_t> col(n), exp(L);
        for (size_t r = 0; r < n; r++) col[r] = t[r][c].value();
        tvmo_lde_column(col.data(), n, exp.data(), L, 7);
        for (size_t r = 0; r < L; r++) ok = ok && lde[r].size() == w && lde[r][c].value() == exp[r];
    }
    expect(ok, "LDE::extend_table 64x7 -> 256");
    expect(LDE::extend_table({}, domain(4, 1), domain(16, 7)).empty(), "LDE::extend_table(empty)");
    expect_throw<std::invalid_argument>(
        [] { LDE::extend_column(rand_vec(12), domain(12, 1), domain(48, 7)); }, "LDE::extend_column(12)");
}

void check_tip5() {
    uint8_t lk[256];
    uint64_t mds[16], rc[80];
    tvmo_tip5_parameters(lk, mds, rc);
    bool ok = true;
    for (int i = 0; i < 256; i++) ok = ok && Tip5::LOOKUP_TABLE[i] == lk[i];
    for (int i = 0; i < 16; i++) ok = ok && (uint64_t)Tip5::MDS_MATRIX_FIRST_COLUMN[i] == mds[i];
    for (int i = 0; i < 80; i++) ok = ok && Tip5::ROUND_CONSTANTS[i].value() == rc[i];
    expect(ok, "Tip5 parameter tables");

    Tip5 a = Tip5::init();
    ok = true;
    for (auto& x : a.state) ok = ok && x.value() == 0;
    expect(ok, "Tip5::init zero state");
    for (auto& x : a.state) x = rand_bfe();
    std::vector<uint64_t> st = raw(std::vector<BFieldElement>(a.state.begin(), a.state.end()));
    Tip5 b = a, c = a;
    a.permutation();
    tvmo_tip5_permutation(st.data());
    expect(same(std::vector<BFieldElement>(a.state.begin(), a.state.end()), st), "Tip5::permutation");
    for (size_t r = 0; r < Tip5::NUM_ROUNDS; r++) b.round(r);
    expect(b.state == a.state, "Tip5::round x5 == permutation");
    auto tr = c.trace();
    ok = tr.size() == Tip5::NUM_ROUNDS + 1 && tr.back() == a.state && c.state == a.state;
    Tip5 d;
    d.state = tr[0];
    for (size_t r = 0; r < Tip5::NUM_ROUNDS && ok; r++) {
        d.round(r);
        ok = d.state == tr[r + 1];
    }
    expect(ok, "Tip5::trace");
    expect_throw<std::invalid_argument>([] { Tip5 t; t.round(5); }, "Tip5::round(5)");

    // sponge: absorb overwrites at most RATE elements, squeeze reads them back
    Tip5 s = Tip5::init();
    auto in = rand_vec(13);
    s.absorb(in);
    std::vector<uint64_t> ss(16, 0);
    for (size_t i = 0; i < 10; i++) ss[i] = in[i].value();
    tvmo_tip5_permutation(ss.data());
    auto sq = s.squeeze(12);
    expect(sq.size() == 10 && same(sq, std::vector<uint64_t>(ss.begin(), ss.begin() + 10)), "Tip5 absorb/squeeze");

    for (size_t len : {0u, 1u, 9u, 10u, 11u, 20u, 264u, 379u}) {
        auto v = rand_vec(len);
        uint64_t exp[5];
        tvmo_hash_varlen(len ? raw(v).data() : nullptr, len, exp);
        expect(same(Tip5::hash_varlen(v), exp), S("Tip5::hash_varlen", len));
        expect(same(hash_row(v), exp) || (len == 0 && hash_row(v) == Digest::zero()), S("hash_row", len));
    }
    std::array<BFieldElement, 10> ten;
    for (auto& x : ten) x = rand_bfe();
    uint64_t e10[5];
    tvmo_hash_10(raw(std::vector<BFieldElement>(ten.begin(), ten.end())).data(), e10);
    expect(same(Tip5::hash_10(ten), e10), "Tip5::hash_10");
    auto l = rand_vec(5), r = rand_vec(5);
    uint64_t ep[5];
    tvmo_hash_pair(raw(l).data(), raw(r).data(), ep);
    expect(same(Tip5::hash_pair(Digest(l[0], l[1], l[2], l[3], l[4]), Digest(r[0], r[1], r[2], r[3], r[4])), ep),
           "Tip5::hash_pair");
}

void check_merkle() {
    for (size_t n : {1u, 2u, 8u, 1024u}) {
        std::vector<uint64_t> lw(5 * n), nodes(10 * n);
        for (auto& x : lw) x = next_u64() % P;
        std::vector<Digest> leaves(n);
        for (size_t i = 0; i < n; i++) leaves[i] = digest_of(&lw[5 * i]);
        tvmo_merkle_build(lw.data(), n, nodes.data());
        MerkleTree t(leaves);
        MerkleTree tp = MerkleTree::parallel_new(leaves);
        expect(same(t.root(), &nodes[5]) && tp.root() == t.root(), S("MerkleTree root", n));
        expect(t.num_leaves() == n && (size_t(1) << t.height()) == n, S("MerkleTree shape", n));
        bool ok = true;
        for (size_t i = 0; i < n; i += (n > 16 ? n / 16 : 1)) {
            ok = ok && t.leaf(i) == leaves[i];
            auto path = t.authentication_path(i);
            ok = ok && path.size() == t.height();
            size_t h = n + i;
            for (size_t k = 0; k < path.size() && ok; k++, h /= 2) ok = same(path[k], &nodes[5 * (h ^ 1)]);
            ok = ok && MerkleTree::verify(t.root(), i, leaves[i], path);
            if (!path.empty()) ok = ok && !MerkleTree::verify(t.root(), i ^ 1, leaves[i], path);
        }
        expect(ok, S("MerkleTree leaf/path/verify", n));
        std::vector<size_t> idx;  // one leaf for n = 1: the reference accepts no other
        for (int q = 0; q < (n == 1 ? 1 : 5); q++) idx.push_back(next_u64() % n);
        auto st = t.authentication_structure(idx);
        std::vector<size_t> eidx(64 * 5);
        const long m = tvmo_auth_structure_indices(n, idx.data(), idx.size(), eidx.data(), eidx.size());
        ok = (long)st.size() == m;
        for (long q = 0; q < m && ok; q++) ok = same(st[q], &nodes[5 * eidx[q]]);
        expect(ok, S("MerkleTree::authentication_structure", n));
        std::vector<Digest> lv;
        for (size_t i : idx) lv.push_back(leaves[i]);
        expect(MerkleTree::verify_authentication_structure(t.root(), n, idx, lv, st),
               S("verify_authentication_structure", n));
        if (n > 1) {
            auto bad = lv;  // every copy of the first leaf altered (a later duplicate would win)
            for (size_t q = 0; q < idx.size(); q++)
                if (idx[q] == idx[0]) bad[q][0] = bad[q][0] + BFieldElement(1);
            expect(!MerkleTree::verify_authentication_structure(t.root(), n, idx, bad, st),
                   S("verify_authentication_structure rejects", n));
        }
        expect_throw<std::out_of_range>([&] { t.leaf(n); }, S("MerkleTree::leaf(n)", n));
        expect_throw<std::out_of_range>([&] { t.authentication_path(n); }, S("authentication_path(n)", n));
    }
    expect_throw<std::invalid_argument>([] { MerkleTree t(std::vector<Digest>{}); }, "MerkleTree(empty)");
    expect_throw<std::invalid_argument>([] { MerkleTree t(std::vector<Digest>(3)); }, "MerkleTree(3)");
    expect(MerkleTree::sibling_index(6) == 7 && MerkleTree::parent_index(7) == 3, "sibling/parent index");
}

// (x^n - t^n) * r(x) added to the interpolant, for one column, on the oracle
std::vector<uint64_t> oracle_rand(const std::vector<BFieldElement>& col, const std::vector<BFieldElement>& r,
                                  size_t L, uint64_t t, uint64_t o, int truncate) {
    std::vector<uint64_t> out(L), rr = raw(r);
    tvmo_lde_randomized_column(raw(col).data(), col.size(), rr.empty() ? nullptr : rr.data(), rr.size(),
                               out.data(), L, t, o, truncate);
    return out;
}

void check_randomized() {
    for (auto [n, R, L, t] : std::vector<std::tuple<size_t, size_t, size_t, uint64_t>>{
             {64, 98, 256, 1}, {8, 3, 32, 5}, {4, 20, 8, 11}, {1, 5, 4, 1}, {1024, 0, 4096, 3}}) {
        auto col = rand_vec(n), r = rand_vec(R);
        auto got = RandomizedLDE::extend_column_with_randomizer(col, domain(n, t), domain(L, 7), r);
        expect(same(got, oracle_rand(col, r, L, t, 7, 0)), S("extend_column_with_randomizer n", n) + S(" R", R));
        // XFE column with a base-field and with an XFE randomizer
        std::vector<XFieldElement> xc(n);
        std::vector<BFieldElement> limb[3];
        for (size_t i = 0; i < n; i++) {
            xc[i] = XFieldElement(rand_bfe(), rand_bfe(), rand_bfe());
            for (int k = 0; k < 3; k++) limb[k].push_back(xc[i].coeff(k));
        }
        auto gx = RandomizedLDE::extend_xfield_column_with_randomizer(xc, domain(n, t), domain(L, 7), r);
        std::vector<XFieldElement> xr(R);
        std::vector<BFieldElement> rl[3];
        for (size_t j = 0; j < R; j++) {
            xr[j] = XFieldElement(rand_bfe(), rand_bfe(), rand_bfe());
            for (int k = 0; k < 3; k++) rl[k].push_back(xr[j].coeff(k));
        }
        auto gxx = RandomizedLDE::extend_xfield_column_with_xfield_randomizer(xc, domain(n, t), domain(L, 7), xr);
        bool ok = gx.size() == L && gxx.size() == L;
        for (int k = 0; k < 3 && ok; k++) {
            auto e1 = oracle_rand(limb[k], k == 0 ? r : std::vector<BFieldElement>(R), L, t, 7, 1);
            auto e2 = oracle_rand(limb[k], rl[k], L, t, 7, 1);
            for (size_t j = 0; j < L && ok; j++) ok = gx[j].coeff(k).value() == e1[j] && gxx[j].coeff(k).value() == e2[j];
        }
        expect(ok, S("extend_xfield_column_with_(x)randomizer n", n) + S(" R", R));
    }
    // zerofier helpers
    auto z = RandomizedLDE::compute_zerofier(domain(16, 7));
    expect(z.size() == 17 && z[16].value() == 1 && z[0].value() == (P - tvmo_pow(7, 16)) % P,
           "compute_zerofier");
    expect(RandomizedLDE::verify_zerofier(domain(16, 7), z), "verify_zerofier(zerofier)");
    BPolynomial notz = z;
    notz[1] = BFieldElement(1);
    expect(!RandomizedLDE::verify_zerofier(domain(16, 7), notz), "verify_zerofier rejects");
    auto r = BPolynomial(rand_vec(5));
    auto zr = RandomizedLDE::mul_zerofier_with(domain(16, 7), r);
    auto zr2 = z * r;
    bool ok = zr.size() == zr2.size();
    for (size_t i = 0; i < zr.size() && ok; i++) ok = zr[i] == zr2[i];
    expect(ok, "mul_zerofier_with == zerofier * r");
    expect_throw<std::invalid_argument>([] { RandomizedLDE::compute_zerofier(domain(0, 7)); }, "compute_zerofier(0)");
    expect_throw<std::domain_error>(
        [] { RandomizedLDE::extend_column_with_randomizer(rand_vec(8), domain(8, 0), domain(32, 7), rand_vec(2)); },
        "extend_column_with_randomizer(trace offset 0)");
}

void check_lde_table() {
    const size_t n = 64, w = 23, L = 256;
    std::vector<std::vector<BFieldElement>> t(n), rnd(w);
    for (auto& r : t) r = rand_vec(w);
    for (size_t c = 0; c < w; c++) rnd[c] = rand_vec(c % 3 == 0 ? 98 : c % 3 == 1 ? 0 : 7);
    auto ext = LDETable::extend_table_with_randomizers(t, domain(n, 1), domain(L, 7), rnd);
    bool ok = ext.size() == L;
    std::vector<uint64_t> rm(L * w);
    for (size_t c = 0; c < w && ok; c++) {
        std::vector<BFieldElement> col(n);
        for (size_t r = 0; r < n; r++) col[r] = t[r][c];
        auto exp = oracle_rand(col, rnd[c], L, 1, 7, 0);
        for (size_t r = 0; r < L; r++) {
            ok = ok && ext[r][c].value() == exp[r];
            rm[r * w + c] = exp[r];
        }
    }
    expect(ok, "LDETable::extend_table_with_randomizers");
    std::vector<uint64_t> leaves(5 * L), nodes(10 * L);
    for (size_t r = 0; r < L; r++) tvmo_hash_varlen(&rm[r * w], w, &leaves[5 * r]);
    tvmo_merkle_build(leaves.data(), L, nodes.data());
    auto [digests, root] = LDETable::compute_merkle_tree(ext);
    ok = digests.size() == L && same(root, &nodes[5]);
    for (size_t r = 0; r < L && ok; r++) ok = same(digests[r], &leaves[5 * r]);
    expect(ok, "LDETable::compute_merkle_tree");
    expect(same(LDETable::compute_lde_and_merkle(t, domain(n, 1), domain(L, 7), rnd), &nodes[5]),
           "LDETable::compute_lde_and_merkle");
    expect(LDETable::compute_lde_and_merkle({}, domain(n, 1), domain(L, 7), {}) == Digest(),
           "compute_lde_and_merkle(empty)");
    expect_throw<std::invalid_argument>(
        [&] { LDETable::extend_table_with_randomizers(t, domain(n, 1), domain(L, 7), {}); },
        "extend_table_with_randomizers(randomizer count)");
}
}  // namespace

int main() {
    check_ntt();
    check_lde();
    check_tip5();
    check_merkle();
    check_randomized();
    check_lde_table();
    std::printf("shim selftest: %d checks, %d failed\n", g_checks, g_failed);
    return g_failed ? 1 : 0;
}
