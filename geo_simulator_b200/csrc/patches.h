// Element-patch layout of the matrix-free operator (host-built).
//
// Elements are ordered along a Morton curve of their vertex centroids and cut
// into patches of at most kPatchElems elements touching at most kPatchNodes
// distinct nodes. Nodes are renumbered in first-touch order over that element
// order, so each patch "owns" one contiguous range of new node ids (the nodes it
// touches first); the other nodes it touches ("foreign") were owned by earlier
// patches and are listed explicitly. Connectivity is stored as 16-bit indices
// into the patch-local node table [own range | foreign list].
#pragma once

#include <cstdint>
#include <vector>

namespace geo {

constexpr int kPatchElems = 384;
constexpr int kPatchNodes = 1024;

// node flag bits (new numbering)
constexpr uint8_t kFlagDir0 = 1;    // component c Dirichlet: kFlagDir0 << c
constexpr uint8_t kFlagShared = 128;  // touched by more than one patch

struct PatchLayout {
    int64_t n_elem = 0, n_nodes = 0;
    int64_t n_patches = 0;
    int max_local = 0;                   // largest patch-local node table
    std::vector<int32_t> eperm;          // new element -> original element
    std::vector<int32_t> nperm;          // new node -> original node
    std::vector<int32_t> ninv;           // original node -> new node
    std::vector<int32_t> patch_elem;     // [n_patches + 1]
    std::vector<int32_t> patch_own;      // [n_patches + 1] new node ids
    std::vector<int32_t> patch_foreign;  // [n_patches + 1] offsets into foreign
    std::vector<int32_t> foreign;        // new node ids, ascending per patch
    std::vector<uint16_t> lconn;         // SoA [10][n_elem] patch-local indices
    std::vector<uint8_t> shared;         // [n_nodes] new ids: 1 if shared
};

// conn: AoS [E][10] original ids; xyz AoS [N][3].
void build_patches(int64_t n_nodes, const double* xyz, int64_t n_elem, const int32_t* conn, PatchLayout& out);

}  // namespace geo
