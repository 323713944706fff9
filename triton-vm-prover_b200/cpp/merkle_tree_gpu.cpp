// triton_vm::MerkleTree and hash_row (include/merkle/merkle_tree.hpp) on the
// GPU, in place of the reference's src/merkle/merkle_tree.cpp.  The tree keeps
// the reference's heap layout in nodes_ (root at 1, leaves at [n, 2n), node 0
// zero), built by the library in one call; paths and structures are gathers
// from it, and verification hashes on the GPU.
#include <algorithm>
#include <cmath>
#include <unordered_map>

#include "merkle/merkle_tree.hpp"
#include "shim.hpp"

namespace triton_vm {

using tvmc_shim::check;
using tvmc_shim::words;

// Same checks and messages as src/merkle/merkle_tree.cpp:12-33.
MerkleTree::MerkleTree(const std::vector<Digest>& leaves) {
    if (leaves.empty()) throw std::invalid_argument("Cannot create Merkle tree with no leaves");
    if ((leaves.size() & (leaves.size() - 1)) != 0)
        throw std::invalid_argument("Number of leaves must be a power of 2");
    num_leaves_ = leaves.size();
    nodes_.resize(2 * num_leaves_);
    std::copy(leaves.begin(), leaves.end(), nodes_.begin() + num_leaves_);
    build_tree();
}

MerkleTree MerkleTree::parallel_new(const std::vector<Digest>& leaves) { return MerkleTree(leaves); }

// Every level in one library call; the leaves are read from nodes_[n, 2n)
// before the tree is written back over nodes_.
void MerkleTree::build_tree() {
    check(tvmc_merkle_tree_heap_host(words(nodes_.data() + num_leaves_), num_leaves_, words(nodes_.data())));
}

Digest MerkleTree::root() const { return nodes_[1]; }

size_t MerkleTree::height() const { return static_cast<size_t>(std::log2(num_leaves_)); }

Digest MerkleTree::leaf(size_t index) const {
    if (index >= num_leaves_) throw std::out_of_range("Leaf index out of range");
    return nodes_[num_leaves_ + index];
}

Digest MerkleTree::node(size_t index) const {
    if (index == 0 || index >= nodes_.size()) throw std::out_of_range("Node index out of range");
    return nodes_[index];
}

size_t MerkleTree::sibling_index(size_t node_index) { return node_index ^ 1; }

size_t MerkleTree::parent_index(size_t node_index) { return node_index / 2; }

std::vector<Digest> MerkleTree::authentication_path(size_t leaf_index) const {
    if (leaf_index >= num_leaves_) throw std::out_of_range("Leaf index out of range");
    std::vector<Digest> path;
    for (size_t i = num_leaves_ + leaf_index; i > 1; i /= 2) path.push_back(nodes_[sibling_index(i)]);
    return path;
}

std::vector<size_t> MerkleTree::authentication_structure_node_indices(size_t num_leaves,
                                                                      const std::vector<size_t>& leaf_indices) {
    if (num_leaves == 0) throw std::invalid_argument("num_leaves must be > 0");
    if ((num_leaves & (num_leaves - 1)) != 0) throw std::invalid_argument("num_leaves must be a power of 2");
    size_t count = 0;
    check(tvmc_auth_structure_indices(num_leaves, leaf_indices.data(), leaf_indices.size(), nullptr, 0, &count));
    std::vector<uint64_t> idx(count);
    check(tvmc_auth_structure_indices(num_leaves, leaf_indices.data(), leaf_indices.size(), idx.data(), count,
                                      &count));
    return std::vector<size_t>(idx.begin(), idx.end());
}

std::vector<Digest> MerkleTree::authentication_structure(const std::vector<size_t>& leaf_indices) const {
    std::vector<Digest> out;
    for (size_t i : authentication_structure_node_indices(num_leaves_, leaf_indices)) out.push_back(nodes_[i]);
    return out;
}

// MerkleTree::verify (src/merkle/merkle_tree.cpp:343-364): the root implied by
// the path, computed on the GPU, against `root`.
bool MerkleTree::verify(const Digest& root, size_t leaf_index, const Digest& leaf,
                        const std::vector<Digest>& auth_path) {
    Digest got;
    check(tvmc_merkle_root_from_paths_host(&leaf_index, words(&leaf), auth_path.empty() ? nullptr : words(auth_path.data()),
                                           1, auth_path.size(), words(&got)));
    return got == root;
}

// MerkleTree::verify_authentication_structure (src/merkle/merkle_tree.cpp:267-341):
// the same acceptance rules; the parents are hashed level by level, each level
// in one batched GPU call.
bool MerkleTree::verify_authentication_structure(const Digest& root, size_t num_leaves,
                                                 const std::vector<size_t>& leaf_indices,
                                                 const std::vector<Digest>& leaves,
                                                 const std::vector<Digest>& auth_structure) {
    if (leaf_indices.size() != leaves.size()) return false;
    if (num_leaves == 0 || (num_leaves & (num_leaves - 1)) != 0) return false;
    if (num_leaves == 1) {
        if (leaf_indices.size() != 1 || leaf_indices[0] != 0) return false;
        return leaves[0] == root;
    }
    std::vector<size_t> auth_indices;
    try {
        auth_indices = authentication_structure_node_indices(num_leaves, leaf_indices);
    } catch (...) {
        return false;
    }
    if (auth_indices.size() != auth_structure.size()) return false;
    std::unordered_map<size_t, Digest> known;
    for (size_t i = 0; i < leaf_indices.size(); ++i) known[num_leaves + leaf_indices[i]] = leaves[i];
    for (size_t i = 0; i < auth_structure.size(); ++i) known[auth_indices[i]] = auth_structure[i];
    // level by level from the leaves: every known pair whose parent is unknown
    for (size_t lo = num_leaves; lo > 1 && !known.count(1); lo /= 2) {
        std::vector<size_t> lefts;
        for (const auto& kv : known)
            if (kv.first >= lo && kv.first < 2 * lo && !(kv.first & 1) && known.count(kv.first + 1) &&
                !known.count(kv.first / 2))
                lefts.push_back(kv.first);
        if (lefts.empty()) continue;
        std::sort(lefts.begin(), lefts.end());
        std::vector<Digest> l(lefts.size()), r(lefts.size()), p(lefts.size());
        for (size_t i = 0; i < lefts.size(); i++) {
            l[i] = known[lefts[i]];
            r[i] = known[lefts[i] + 1];
        }
        check(tvmc_hash_pairs_host(words(l.data()), words(r.data()), words(p.data()), lefts.size()));
        for (size_t i = 0; i < lefts.size(); i++) known[lefts[i] / 2] = p[i];
    }
    auto it = known.find(1);
    return it != known.end() && it->second == root;
}

// hash_row (src/merkle/merkle_tree.cpp:366-373): the empty row hashes to zero.
Digest hash_row(const std::vector<BFieldElement>& row) {
    if (row.empty()) return Digest::zero();
    return Tip5::hash_varlen(row);
}

}  // namespace triton_vm
