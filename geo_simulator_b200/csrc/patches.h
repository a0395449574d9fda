// Element-patch layout of the matrix-free operator (built on the GPU).
//
// Elements are ordered along a Morton curve of their vertex centroids and cut
// into patches of kPatchElems consecutive elements. Nodes are renumbered in
// first-touch order over that element order, so each patch "owns" one
// contiguous range of new node ids (the nodes it touches first); the other
// nodes it touches ("foreign") were owned by earlier patches and are listed
// explicitly. Connectivity is stored as 16-bit indices into the patch-local
// node table [own range | foreign list].
#pragma once

#include <cstdint>

#include "common.cuh"

namespace geo {

constexpr int kPatchElems = 384;

// Shared-memory slot of patch-local node u in the patch kernels' node tables:
// one unused word after every 32 nodes. First-touch numbering places the nodes
// that a warp's 32 elements read in one access at strides that share banks; the
// padding spreads them (an emulation of the layout on a structured cube: 4.2 ->
// 2.8 shared-memory wavefronts per warp access of the element phase). The 16-bit
// local connectivity holds slots; loops over a patch's nodes map u -> slot.
__host__ __device__ constexpr int patch_slot(int u) { return u + (u >> 5); }

// node flag bits (patch numbering)
constexpr uint8_t kFlagDir0 = 1;      // component c is Dirichlet: kFlagDir0 << c
constexpr uint8_t kFlagShared = 128;  // touched by more than one patch

struct PatchLayout {
    int64_t n_elem = 0, n_nodes = 0;
    int n_patches = 0;
    int max_local = 0;          // largest patch-local node table, in slots (patch_slot)
    DevBuf<int32_t> eperm;      // new element -> original element
    DevBuf<int32_t> nperm;      // new node -> original node
    DevBuf<int32_t> ninv;       // original node -> new node
    DevBuf<int32_t> patch_elem;     // [n_patches + 1]
    DevBuf<int32_t> patch_own;      // [n_patches + 1] new node ids
    DevBuf<int32_t> patch_foreign;  // [n_patches + 1] offsets into foreign
    DevBuf<int32_t> foreign;        // new node ids, ascending per patch
    // Patch-major local connectivity, two 16-bit indices per word:
    // lc[(p * 5 + l / 2) * kPatchElems + j] holds, in bits 16*(l%2).., the
    // slot (patch_slot) of local node l of the patch's element j (entries
    // past a short last patch are 0). Within a patch, elements are ordered so that
    // every aligned group of 32 (one warp) shares no node where possible.
    DevBuf<uint32_t> lc;            // [n_patches][5][kPatchElems]
    DevBuf<uint8_t> shared;         // [n_nodes] patch numbering: 1 if shared
};

// xyz: device SoA [3][N]; conn: device SoA [10][E] (original numbering).
void build_patches(cudaStream_t s, int64_t n_nodes, const double* xyz, int64_t n_elem, const int32_t* conn,
                   PatchLayout& out);

}  // namespace geo
