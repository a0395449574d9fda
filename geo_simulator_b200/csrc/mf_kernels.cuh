// Kernels of the matrix-free operator and its PCG (see matfree.cu).
//
// Patch apply (k_patch): a CTA works through whole patches (patch = blockIdx.x,
// += gridDim.x). The patch's element data (16-bit local connectivity and the
// per-element qdata, contiguous per patch), its foreign node ids and flags
// (aligned per-patch segments) and its sizes are brought into shared memory with
// cp.async.bulk (bulk copy engine, mbarrier completion), double-buffered so the
// next patch's copy is in flight while the current one is processed; the gather
// then needs a single round trip to global memory. Per patch:
//   1. gather: every patch-local node's input value is read once from global
//      memory into a shared table (own nodes form one contiguous range);
//   2. element pass: each thread applies K_e to its elements from the shared
//      table and accumulates into a shared output table with shared atomics
//      (exact INT32 fixed point for FP32, see Scatter). Elements are ordered so
//      a warp's 32 elements share no node, so these atomics do not collide;
//   3. flush: a plain store for nodes no other patch touches, red.global.add
//      for the shared ones. In "halo" mode (every mode, when the operator has
//      halo slots) every own node is a plain store and every foreign node a
//      plain store to its own slot of a halo array; the slots are numbered by
//      owner node, so the node update (PCG) or k_halo_combine (operator apply,
//      lift) adds a node's foreign contributions from consecutive slots in a
//      fixed order. No global atomics are issued and results are bit-identical
//      from run to run.
// In PCG mode step 1 also forms the new search direction p = z + beta p_old
// (z = D^-1 r) on the fly: the Jacobi scaling and the p-update ride on the
// operator's gather. p is double-buffered by iteration parity.
//
// PCG node update (k_pcg_update): x += alpha p, r -= alpha q (Dirichlet rows
// q = char_diag p), z = D^-1 r, and the r.r / r.z partial sums; loads are
// issued for several entries before any store so they overlap.
//
// Every reduction is single pass: each block writes its partial, the last block
// to finish (ticket counter) sums the partials in a fixed order and updates the
// device-resident PcgState, which the next kernel reads. No host round trip per
// iteration and no grid-wide spin wait.
#pragma once

#include <type_traits>

#include "matfree.cuh"
#include "patches.h"

namespace geo {

constexpr int kPatchBS = 192;  // threads of the patch kernel (2 elements each)
constexpr int kNodeBS = 256;   // threads of the node kernels
constexpr int kUnroll = 4;     // entries in flight per thread in the node kernels
constexpr int kGather = 4;     // patch-local nodes in flight per thread in the gather

enum : int { MODE_FREE = 0, MODE_LIFT = 1, MODE_PCG = 2 };
enum : int { ST_DONE = 1, ST_REFRESH = 2, ST_CONVERGED = 4, ST_BREAKDOWN = 8 };
enum : int { TICKET_PATCH = 0, TICKET_UPDATE = 1, TICKET_AUX = 2 };

struct PatchMeta;

struct PatchView {
    int64_t E, N;
    int n_patches, max_local, dpn;
    const int32_t* pe;
    const int32_t* po;
    const int32_t* pf;
    const int32_t* foreign;
    const uint32_t* lc;  // patch-major paired connectivity [P][5][kPatchElems]
    const uint8_t* flags;
    // scatter bound per patch (see Scatter): (max element incidences of a
    // patch-local node) x max_e ||K_e||_inf x 1.001, rounded up
    const float* bound32;
    // foreign ids and flags again, in per-patch segments that start at pfa[p]
    // (multiples of kForeignAlign entries) so that they travel with the patch's
    // bulk copy; max_for = the largest foreign count of a patch
    const int32_t* pfa;
    const int32_t* fids;
    const uint8_t* fflags;
    int max_for;
    int max_own;   // the largest own-node count of a patch
    int own_bulk;  // own-node slices by bulk copy (FP32 thermal PCG; the launch's shared memory holds them)
    // halo mode (PCG): the halo slot of every foreign entry, in
    // the same per-patch segments as fids. halo: 0 off; 1 the slots ride in the
    // patch's bulk copy; 2 the flush reads them from global memory (coalesced), for
    // launches where the shared-memory copy would cost a resident block
    const int32_t* fslot;
    int halo;
    // per patch: element count, own range, foreign count and segment start, scatter
    // bound, as one 32-byte record (16-byte aligned), so that the patch kernel's
    // copy issue needs one prefetched record instead of dependent global loads
    const PatchMeta* rec;
};

// ------------------------------------------------------------------ shared-memory scatter
// Element contributions are accumulated in shared memory as exact integers.
// Every contribution c of a patch is scaled by a power of two S chosen so that
// the sum of all contributions to one DOF stays below kLim, then rounded to an
// integer held in kWords INT32 words. Integer sums are exact, so the
// accumulation does not depend on the order of the atomics, and INT32 shared
// atomics cost a fraction of FP32 / FP64 ones (on B200, random banks: about 3.7
// SM cycles per warp operation against 13.4 for FP32 and 22 for FP64).
// The bound behind S is rigorous: K_e annihilates constants (thermal) and
// rigid translations (elasticity), so |(K_e x)_i| <= ||K_e||_inf * max_c h_c,
// h_c = half the range of component c of x over the patch; a margin of 2^-16
// max|x| covers the rounding of the apply, and the patch's largest number of
// element incidences per node bounds the sum (PatchView::bound32).
// FP32: one word (|sum| < 2^30, resolution 2^-30 of the bound). FP64: three
// words holding hi 2^42 + mid 2^21 + lo (|sum| < 2^62, resolution 2^-62 of the
// bound, below the FP64 rounding of the result). Word w of DOF slot s sits at
// acc[w * m + s].
template <class T>
struct Scatter;

template <>
struct Scatter<float> {
    static constexpr float kLim = 1073741824.0f;  // 2^30
    static constexpr int kLimExp = 30;
    static constexpr int kWords = 1;
    __device__ __forceinline__ static void zero(int* acc, int, int slot) { acc[slot] = 0; }
    __device__ __forceinline__ static void add(int* acc, int, int slot, float v) {
        atomicAdd(acc + slot, __float2int_rn(v));
    }
    __device__ __forceinline__ static float get(const int* acc, int, int slot) { return (float)acc[slot]; }
    // read and clear (the flush leaves the table zero for the next patch)
    __device__ __forceinline__ static float take(int* acc, int, int slot) {
        const int v = acc[slot];
        acc[slot] = 0;
        return (float)v;
    }
};

template <>
struct Scatter<double> {
    static constexpr float kLim = 4.611686018427388e18f;  // 2^62
    static constexpr int kLimExp = 62;
    static constexpr int kWords = 3;
    __device__ __forceinline__ static void zero(int* acc, int m, int slot) {
        acc[slot] = 0;
        acc[m + slot] = 0;
        acc[2 * m + slot] = 0;
    }
    // v = hi 2^42 + mid 2^21 + lo; hi and mid are exact, lo rounds the last fraction
    __device__ __forceinline__ static void add(int* acc, int m, int slot, double v) {
        const int hi = __double2int_rn(v * 2.2737367544323206e-13);  // 2^-42
        const double r = fma(-(double)hi, 4398046511104.0, v);         // 2^42, exact
        const int mid = __double2int_rn(r * 4.76837158203125e-07);    // 2^-21
        const int lo = __double2int_rn(fma(-(double)mid, 2097152.0, r));
        atomicAdd(acc + slot, hi);
        atomicAdd(acc + m + slot, mid);
        atomicAdd(acc + 2 * m + slot, lo);
    }
    __device__ __forceinline__ static double get(const int* acc, int m, int slot) {
        return fma((double)acc[slot], 4398046511104.0, fma((double)acc[m + slot], 2097152.0, (double)acc[2 * m + slot]));
    }
    __device__ __forceinline__ static double take(int* acc, int m, int slot) {
        const double v = get(acc, m, slot);
        zero(acc, m, slot);
        return v;
    }
};

// S = the largest power of two <= 2^lim_exp / bx, clamped to [2^-100, 2^100], and
// 1/S, both exact, from the exponent field of bx > 0 (no division): with
// bx = m 2^e, m in [1, 2), S = 2^(lim_exp - e) when m = 1, else 2^(lim_exp - e - 1);
// a subnormal bx gives the upper clamp, an infinite one the lower.
__device__ __forceinline__ void pow2_scale(float bx, int lim_exp, float& S, float& invS) {
    const unsigned bits = __float_as_uint(bx);
    const int ef = (int)(bits >> 23);
    int se = lim_exp - (ef - 127) - ((bits & 0x7fffffu) != 0u ? 1 : 0);
    if (ef == 0) se = 100;
    if (ef == 255) se = -100;
    se = min(max(se, -100), 100);
    S = __uint_as_float((unsigned)(se + 127) << 23);
    invS = __uint_as_float((unsigned)(127 - se) << 23);
}

// float <-> unsigned key with the same order (for warp min/max reductions)
__device__ __forceinline__ unsigned float_key(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Device-resident PCG scalars.
struct PcgState {
    double rz, rz_old, pAp, alpha, beta, bnorm, s_scale, rmax, res, ratio, s_new;
    double tol, abs_tol, delta, cd;
    long long it, max_it, nupd;
    int flags;
    int err;  // DEV_ERR_* bits raised by bounded waits
    unsigned int ticket[4];
};

template <class T>
struct PatchArgs {
    const T* x;  // FREE / LIFT input
    T* y;        // output (free rows)
    // PCG mode
    const T* r;
    const T* dinv;
    T* pbuf0;
    T* pbuf1;
    PcgState* st;
    double* part;  // [gridDim.x][2]
    int* err;      // DEV_ERR_* bits (bounded waits)
    T* halo;       // halo mode: foreign contributions by slot (DPN values each)
    T* xsol;       // PCG z-form: the FP32 solution correction, updated on the own nodes
};

// ------------------------------------------------------------------ bulk copy + mbarrier
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// global -> shared bulk copy (no multicast); dst/src 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait (2 s of %globaltimer); returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_timer_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_timer_ns() - t0 > 2000000000ull) return false;
    return true;
}

// Last-block detection after every block stored its partial.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (s_last) __threadfence();
    return s_last != 0;
}

// bytes of one patch's element data (connectivity + qdata), 16-byte multiple
template <class K, class T>
__host__ __device__ constexpr uint32_t patch_bytes_lc() { return 5 * kPatchElems * 4; }
template <class K, class T>
__host__ __device__ constexpr uint32_t patch_bytes_qd() { return K::NQD * kPatchElems * (uint32_t)sizeof(T); }

constexpr int kForeignAlign = 16;  // foreign segments start at multiples of 16 entries

__host__ __device__ inline uint32_t round16(uint32_t b) { return (b + 15u) & ~15u; }

// A patch's sizes, written by the issuing thread next to its bulk copies.
struct __align__(16) PatchMeta {
    int n_el, o0, nown, nfor, fa;
    float bound;  // PatchView::bound32 of the patch
    int pad0, pad1;
};

// PatchView::rec from the per-patch offsets and bounds
__global__ void k_patch_records(PatchView pv, PatchMeta* __restrict__ rec) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pv.n_patches) return;
    PatchMeta m;
    m.n_el = pv.pe[p + 1] - pv.pe[p];
    m.o0 = pv.po[p];
    m.nown = pv.po[p + 1] - m.o0;
    m.nfor = pv.pf[p + 1] - pv.pf[p];
    m.fa = pv.pfa[p];
    m.bound = pv.bound32[p];
    m.pad0 = m.pad1 = 0;
    rec[p] = m;
}

// 16-byte asynchronous copy global -> shared (cp.async, no bulk); completes at cp_async_wait_all
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// per-buffer bytes of [meta | foreign ids | foreign flags | halo slots (halo == 1)]
__host__ __device__ inline uint32_t patch_aux_ids(int max_for) {
    return round16((uint32_t)((max_for + kForeignAlign - 1) / kForeignAlign * kForeignAlign) * 4u);
}
__host__ __device__ inline uint32_t patch_aux_flags(int max_for) {
    return round16((uint32_t)((max_for + kForeignAlign - 1) / kForeignAlign * kForeignAlign));
}
__host__ __device__ inline uint32_t patch_aux_bytes(int max_for, int halo) {
    return (uint32_t)sizeof(PatchMeta) + patch_aux_ids(max_for) + patch_aux_flags(max_for) +
           (halo == 1 ? patch_aux_ids(max_for) : 0u);
}

// Own-node slices (PCG mode): D^-1, r and p_old over the patch's own DOF range
// [dpn o0, dpn o1) (components interleaved, so the range is contiguous) and the
// flags of its own nodes, copied with cp.async.bulk from 16-byte aligned starts
// (ranges rounded outwards to 16 bytes). Capacities: values per array, flag bytes.
template <class T>
__host__ __device__ inline uint32_t own_cap(int max_own, int dpn) {
    constexpr uint32_t V = 16 / sizeof(T);
    return ((uint32_t)(max_own * dpn) + 2 * V + V - 1) & ~(V - 1);
}
__host__ __device__ inline uint32_t own_capf(int max_own) { return (uint32_t)(max_own + 32 + 15) & ~15u; }
template <class T>
__host__ __device__ inline uint32_t own_bytes(int max_own, int dpn) {
    return 3u * own_cap<T>(max_own, dpn) * (uint32_t)sizeof(T) + own_capf(max_own);
}
template <class K, class T, int MODE>
__host__ __device__ constexpr bool own_bulk() {
    return MODE == MODE_PCG;
}

// Loop shape of the double-buffered patch kernel.
// - Early (FP32 thermal): the next patch's copy is issued at the top of the loop,
//   a whole patch ahead, and a block barrier after the flush frees the buffer it
//   overwrites. Its gather is short next to the copy's latency.
// - Late (the others): the copy is issued after the gather barrier, when every warp
//   has left the previous flush. No barrier follows the flush, so fast warps start
//   the next gather while others still flush; the node flags then need one table
//   per patch parity.
template <class K, class T, int NBUF>
__host__ __device__ constexpr bool patch_late() {
    return NBUF == 2 && !(K::DPN == 1 && sizeof(T) == 4);
}
template <class K, class T, int NBUF>
__host__ __device__ constexpr int patch_flag_tables() {
    return patch_late<K, T, NBUF>() ? 2 : 1;
}

// shared memory layout: [3 mbarriers (32 B) | NBUF x (lc | qd) | NBUF x (meta | foreign ids | foreign flags) |
// xs | ys | flags (one table, two in the late shape) | own-node slices (PCG)]
template <class K, class T, int NBUF>
__host__ __device__ constexpr size_t patch_smem_fixed() {
    return 32 + (size_t)NBUF * (patch_bytes_lc<K, T>() + patch_bytes_qd<K, T>());
}
template <class K, class T, int NBUF>
__host__ __device__ inline size_t patch_smem_tables(int max_for, int halo) {
    return patch_smem_fixed<K, T, NBUF>() + (size_t)NBUF * patch_aux_bytes(max_for, halo);
}

// Resident blocks per SM the register allocation must allow (the minimum-blocks
// argument of the launch bounds): FP32 elasticity and FP64 thermal 2, FP64
// elasticity 1, as many as their shared memory allows on the bench meshes. FP32
// thermal gets no target (0): it compiles to 79-80 registers, 4 blocks of 192
// threads, by itself, and a target of 4 made the same register count run 2% slower.
template <class K, class T>
__host__ __device__ constexpr int patch_min_blocks() {
    return sizeof(T) == 4 ? (K::DPN == 1 ? 0 : 2) : (K::DPN == 1 ? 2 : 1);
}

// HG = 1: the halo-mode variant whose flush reads the halo slots from global
// memory (PatchView::halo == 2); HG = 0 serves every other launch.
template <class K, class T, int MODE, int NBUF, int HG = 0>
__global__ void __launch_bounds__(kPatchBS, patch_min_blocks<K, T>())
    k_patch(PatchView pv, const T* __restrict__ qd_all, T cl, T cm, PatchArgs<T> a) {
    constexpr int DPN = K::DPN;
    constexpr uint32_t LCB = patch_bytes_lc<K, T>(), QDB = patch_bytes_qd<K, T>();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // [0..NBUF): element data; [2]: own-node slices
    unsigned char* ebuf = smem + 32;
    const bool OWNB = own_bulk<K, T, MODE>() && pv.own_bulk != 0;
    using SC = Scatter<T>;
    const int M = pv.max_local * DPN;  // DOF slots of the patch-local table (nodes by patch_slot)
    unsigned char* abuf = smem + patch_smem_fixed<K, T, NBUF>();  // NBUF x (meta | ids | flags)
    const bool HALO = HG != 0 || pv.halo != 0;
    const int HMODE = !HALO ? 0 : (HG ? 2 : 1);  // 1: slots in shared memory, 2: from global
    const uint32_t AUX = patch_aux_bytes(pv.max_for, HMODE), AIDS = patch_aux_ids(pv.max_for);
    const uint32_t AFL = patch_aux_flags(pv.max_for);
    T* xs = reinterpret_cast<T*>(smem + patch_smem_tables<K, T, NBUF>(pv.max_for, HMODE));
    int* ys = reinterpret_cast<int*>(xs + M);  // fixed-point accumulators, SC::kWords x M words
    // FP32 scatter: per component, min and max of x over the patch as order keys, by patch parity
    __shared__ unsigned s_lo[2][DPN], s_hi[2][DPN];
    constexpr bool LATE = patch_late<K, T, NBUF>();
    // node flags; in the late shape by patch parity, since the flush of one patch
    // reads them while faster warps already gather the next one
    uint8_t* sfl0 = reinterpret_cast<uint8_t*>(ys + SC::kWords * M);
    const uint32_t OCAP = own_cap<T>(pv.max_own, DPN);
    T* own_d = reinterpret_cast<T*>(
        smem + (((size_t)(sfl0 + patch_flag_tables<K, T, NBUF>() * pv.max_local - smem) + 15) & ~(size_t)15));
    T* own_r = own_d + OCAP;
    T* own_p = own_r + OCAP;
    uint8_t* own_f = reinterpret_cast<uint8_t*>(own_p + OCAP);
    // Preconditioned-residual form of the mixed solver's FP32 PCG (thermal and elasticity):
    // the node update keeps z = D^-1 r (a.r holds z) instead of r, so the gather
    // forms p = z + beta p_old from two vectors, and the solution update
    // x += alpha_prev p_old of the previous iteration rides here, on the own nodes'
    // p_old (a.xsol holds the FP32 solution). The FP64 drop-in keeps the
    // reference's form (iterative.rs:46-119).
    constexpr bool ZF = MODE == MODE_PCG && std::is_same<T, float>::value;
    T beta = T(0), alpha_prev = T(0);
    const T* pold = nullptr;
    T* pnew = nullptr;
    if (MODE == MODE_PCG) {
        if (a.st->flags & (ST_DONE | ST_REFRESH)) return;
        beta = (T)a.st->beta;
        if (ZF) alpha_prev = (T)a.st->alpha;
        const bool odd = a.st->it & 1;
        pold = odd ? a.pbuf1 : a.pbuf0;
        pnew = odd ? a.pbuf0 : a.pbuf1;
    }
    if (threadIdx.x == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&bar[b], 1);
        if (OWNB) mbar_init(&bar[2], 1);
        mbar_fence_init();
        for (int c = 0; c < DPN; ++c) {
            s_lo[0][c] = s_lo[1][c] = 0xffffffffu;
            s_hi[0][c] = s_hi[1][c] = 0u;
        }
    }
    // the accumulators start at zero; each flush clears what it reads
    for (int i = threadIdx.x; i < SC::kWords * M; i += blockDim.x) ys[i] = 0;
    __syncthreads();
    // Thread 0 issues the copies of patch q_j (the block's j-th patch) from its record
    // in s_rec[j & 1], prefetched by cp.async when q_(j-1) was issued, so that no
    // issue waits on a global load.
    __shared__ PatchMeta s_rec[2];
    auto prefetch_rec = [&](int patch, int slot) {
        cp_async16(&s_rec[slot], pv.rec + patch);
        cp_async16(reinterpret_cast<unsigned char*>(&s_rec[slot]) + 16,
                   reinterpret_cast<const unsigned char*>(pv.rec + patch) + 16);
        cp_async_commit();
    };
    // thread 0: the patch's element data, sizes, foreign ids and foreign flags into buffer b
    auto issue = [&](const PatchMeta& m, int patch, int b) {
        unsigned char* ab = abuf + (size_t)b * AUX;
        *reinterpret_cast<PatchMeta*>(ab) = m;  // published by the arrive below
        const uint32_t ib = round16((uint32_t)m.nfor * 4u), fb = round16((uint32_t)m.nfor);
        unsigned char* dst = ebuf + (size_t)b * (LCB + QDB);
        mbar_expect_tx(&bar[b], LCB + QDB + ib + fb + (HMODE == 1 ? ib : 0u));
        bulk_g2s(dst, pv.lc + (size_t)patch * 5 * kPatchElems, LCB, &bar[b]);
        bulk_g2s(dst + LCB, qd_all + (size_t)patch * K::NQD * kPatchElems, QDB, &bar[b]);
        if (ib) {
            bulk_g2s(ab + sizeof(PatchMeta), pv.fids + m.fa, ib, &bar[b]);
            bulk_g2s(ab + sizeof(PatchMeta) + AIDS, pv.fflags + m.fa, fb, &bar[b]);
            if (HMODE == 1) bulk_g2s(ab + sizeof(PatchMeta) + AIDS + AFL, pv.fslot + m.fa, ib, &bar[b]);
        }
    };
    // thread 0: D^-1, r, p_old and flags of the patch's own nodes (single buffer, bar[2])
    auto issue_own = [&](const PatchMeta& m) {
        constexpr int V = 16 / (int)sizeof(T);  // values per 16 bytes
        const int o0 = m.o0, o1 = m.o0 + m.nown;
        const int a0 = (DPN * o0) & ~(V - 1), nv = ((DPN * o1 + V - 1) & ~(V - 1)) - a0;  // 16-byte aligned
        const int f0 = o0 & ~15, nf = ((o1 + 15) & ~15) - f0;                             // flags, 16-byte aligned
        const uint32_t vb = (uint32_t)nv * (uint32_t)sizeof(T);
        mbar_expect_tx(&bar[2], 3u * vb + (uint32_t)nf);
        if (nv) {  // z-form: z, p_old, x in the three slices; else D^-1, r, p_old
            bulk_g2s(own_d, ZF ? a.r + a0 : a.dinv + a0, vb, &bar[2]);
            bulk_g2s(own_r, ZF ? pold + a0 : a.r + a0, vb, &bar[2]);
            bulk_g2s(own_p, ZF ? a.xsol + a0 : pold + a0, vb, &bar[2]);
        }
        if (nf) bulk_g2s(own_f, pv.flags + f0, (uint32_t)nf, &bar[2]);
    };
    if (threadIdx.x == 0 && blockIdx.x < pv.n_patches) {
        const PatchMeta m0 = pv.rec[blockIdx.x];
        issue(m0, blockIdx.x, 0);
        if (OWNB) issue_own(m0);
        if (blockIdx.x + gridDim.x < pv.n_patches) prefetch_rec(blockIdx.x + gridDim.x, 1);
    }
    // thread 0: patch + gridDim.x (the block's (k+1)-th) into buffer b from its prefetched
    // record, and the record after it into the slot just read from
    auto issue_next = [&](int patch, int k, int b) {
        cp_async_wait_all();
        const PatchMeta m = s_rec[(k + 1) & 1];
        issue(m, patch + gridDim.x, b);
        if (patch + 2 * (int)gridDim.x < pv.n_patches) prefetch_rec(patch + 2 * gridDim.x, k & 1);
    };
    uint32_t phase = 0;  // bit b = parity of buffer b; bit 2 = parity of the own-node buffer
    // bit b: a copy into buffer b is in flight (tracked by thread 0, which issues them)
    uint32_t pend = blockIdx.x < pv.n_patches ? (OWNB ? 5u : 1u) : 0u;
    double dot = 0.0, pdd = 0.0;
    int k = 0;
    for (int patch = blockIdx.x; patch < pv.n_patches; patch += gridDim.x, ++k) {
        const int b = NBUF == 2 ? (k & 1) : 0;
        const bool has_next = patch + (int)gridDim.x < pv.n_patches;
        if (!LATE && NBUF == 2 && threadIdx.x == 0 && has_next) {
            issue_next(patch, k, b ^ 1);
            pend |= 1u << (b ^ 1);
        }
        // The patch's sizes, element data and foreign lists. No block barrier here: a
        // thread whose bounded wait ran out skips the gather, and the gather barrier
        // below ends the block.
        bool ok = mbar_wait(&bar[b], (phase >> b) & 1);
        if (ok) {
            phase ^= 1u << b;
            pend &= ~(1u << b);
        }
        if (OWNB) {
            const bool ok2 = mbar_wait(&bar[2], (phase >> 2) & 1);
            if (ok2) {
                phase ^= 4u;
                pend &= ~4u;
            }
            ok = ok && ok2;
        }
        uint8_t* sfl = sfl0 + (LATE ? (k & 1) * pv.max_local : 0);
        const unsigned char* ab = abuf + (size_t)b * AUX;
        const PatchMeta pm = *reinterpret_cast<const PatchMeta*>(ab);
        const int* __restrict__ sfor = reinterpret_cast<const int*>(ab + sizeof(PatchMeta));
        const uint8_t* __restrict__ sffl = ab + sizeof(PatchMeta) + AIDS;
        const int* __restrict__ sfsl = reinterpret_cast<const int*>(ab + sizeof(PatchMeta) + AIDS + AFL);
        const int n_el = pm.n_el, o0 = pm.o0, nown = pm.nown, nloc = nown + pm.nfor;
        const float pbound = pm.bound;
        float xlo[DPN], xhi[DPN];
#pragma unroll
        for (int c = 0; c < DPN; ++c) {
            xlo[c] = 3.0e38f;
            xhi[c] = -3.0e38f;
        }
        // 1. gather (overlaps the bulk copies in flight); each thread issues the
        //    loads of up to kGather nodes before any store
        const int nloc_g = ok ? nloc : 0;
        for (int u0 = threadIdx.x; u0 < nloc_g; u0 += kGather * blockDim.x) {
            int node[kGather];
            uint8_t fl[kGather];
            T d0[kGather][DPN], d1[kGather][DPN], d2[kGather][DPN];
#pragma unroll
            for (int g = 0; g < kGather; ++g) {
                const int u = u0 + g * blockDim.x;
                node[g] = u < nown ? o0 + u : (u < nloc ? sfor[u - nown] : 0);
            }
#pragma unroll
            for (int g = 0; g < kGather; ++g) {
                const int u = u0 + g * blockDim.x;
                if (OWNB && u < nown) {  // from the own-node slices in shared memory
                    fl[g] = own_f[(o0 & 15) + u];
                    const int base = ((DPN * o0) & (16 / (int)sizeof(T) - 1)) + DPN * u;
#pragma unroll
                    for (int c = 0; c < DPN; ++c) {
                        d0[g][c] = own_d[base + c];
                        d1[g][c] = own_r[base + c];
                        d2[g][c] = own_p[base + c];
                    }
                } else if (u < nloc) {
                    fl[g] = u < nown ? pv.flags[node[g]] : sffl[u - nown];
#pragma unroll
                    for (int c = 0; c < DPN; ++c) {
                        const int64_t idx = (int64_t)node[g] * DPN + c;
                        if (ZF) {
                            d0[g][c] = a.r[idx];
                            d1[g][c] = pold[idx];
                            d2[g][c] = u < nown ? a.xsol[idx] : T(0);
                        } else if (MODE == MODE_PCG) {
                            d0[g][c] = a.dinv[idx];
                            d1[g][c] = a.r[idx];
                            d2[g][c] = pold[idx];
                        } else {
                            d0[g][c] = a.x[idx];
                        }
                    }
                }
            }
#pragma unroll
            for (int g = 0; g < kGather; ++g) {
                const int u = u0 + g * blockDim.x;
                if (u >= nloc) continue;
                sfl[u] = fl[g];
#pragma unroll
                for (int c = 0; c < DPN; ++c) {
                    const bool dir = (fl[g] >> c) & 1;
                    T v;
                    if (MODE == MODE_PCG) {
                        const T pn = ZF ? d0[g][c] + beta * d1[g][c] : d0[g][c] * d1[g][c] + beta * d2[g][c];
                        if (u < nown) {
                            pnew[(int64_t)node[g] * DPN + c] = pn;
                            if (ZF) a.xsol[(int64_t)node[g] * DPN + c] = d2[g][c] + alpha_prev * d1[g][c];
                            if (dir) pdd += (double)(pn * pn);
                        }
                        v = dir ? T(0) : pn;
                    } else {
                        v = d0[g][c];
                        if (MODE == MODE_FREE ? dir : !dir) v = T(0);
                    }
                    xs[patch_slot(u) * DPN + c] = v;
                    xlo[c] = fminf(xlo[c], (float)v);
                    xhi[c] = fmaxf(xhi[c], (float)v);
                }
            }
        }
        {
#pragma unroll
            for (int c = 0; c < DPN; ++c) {
                const unsigned lo = __reduce_min_sync(0xffffffffu, float_key(xlo[c]));
                const unsigned hi = __reduce_max_sync(0xffffffffu, float_key(xhi[c]));
                if ((threadIdx.x & 31) == 0) {
                    atomicMin(&s_lo[k & 1][c], lo);
                    atomicMax(&s_hi[k & 1][c], hi);
                }
            }
        }
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicOr(a.err, DEV_ERR_TIMEOUT);
                // let copies still in flight land (bounded waits) before the block's shared memory is released
                for (int q = 0; q < 3; ++q)
                    if ((pend >> q) & 1) mbar_wait(&bar[q], (phase >> q) & 1);
                cp_async_wait_all();
            }
            return;
        }
        // Every warp has left the previous patch's flush: in the late shape its buffer
        // takes the next patch's copy; the own-node buffer (read by the gather only)
        // takes the next patch's slices, during steps 2 and 3.
        if (threadIdx.x == 0 && has_next) {
            if (LATE) {
                issue_next(patch, k, b ^ 1);
                pend |= 1u << (b ^ 1);
            }
            if (OWNB) {
                // The record of patch + gridDim.x is in its slot: issue_next of this patch
                // waited for it (two buffers), or the previous patch's prefetched it (one
                // buffer). Waiting in the first case would wait for the prefetch just issued.
                if (NBUF == 1) cp_async_wait_all();
                issue_own(s_rec[(k + 1) & 1]);
                pend |= 4u;
            }
        }
        // 2. elements, scattered as fixed-point integers with scale S (see Scatter)
        T S = T(1), invS = T(1);
        {
            float half = 0.0f, mabs = 0.0f;
#pragma unroll
            for (int c = 0; c < DPN; ++c) {
                const float lo = key_float(s_lo[k & 1][c]), hi = key_float(s_hi[k & 1][c]);
                if (hi >= lo) {
                    half = fmaxf(half, __fmul_ru(__fsub_ru(hi, lo), 0.5f));
                    mabs = fmaxf(mabs, fmaxf(fabsf(lo), fabsf(hi)));
                }
            }
            const float bx = __fmul_ru(pbound, __fmaf_ru(mabs, 1.52587890625e-05f, half));  // 2^-16
            if (bx > 0.0f) {
                float sf, isf;
                pow2_scale(bx, SC::kLimExp, sf, isf);
                S = (T)sf;
                invS = (T)isf;
            }
            if (threadIdx.x < DPN) {  // next read by the patch after next
                s_lo[(k + 1) & 1][threadIdx.x] = 0xffffffffu;
                s_hi[(k + 1) & 1][threadIdx.x] = 0u;
            }
        }
        const uint32_t* lcs = reinterpret_cast<const uint32_t*>(ebuf + (size_t)b * (LCB + QDB));
        const T* qds = reinterpret_cast<const T*>(ebuf + (size_t)b * (LCB + QDB) + LCB);
        for (int el = threadIdx.x; el < n_el; el += blockDim.x) {
            int li[10];
            T xe[10 * DPN], ye[10 * DPN];
#pragma unroll
            for (int l2 = 0; l2 < 5; ++l2) {
                const uint32_t w = lcs[l2 * kPatchElems + el];
                li[2 * l2] = (int)(w & 0xffffu);
                li[2 * l2 + 1] = (int)(w >> 16);
            }
#pragma unroll
            for (int l = 0; l < 10; ++l)
#pragma unroll
                for (int c = 0; c < DPN; ++c) xe[l * DPN + c] = xs[li[l] * DPN + c];
            K::apply(qds + el, kPatchElems, cl, cm, xe, ye);
            if (MODE == MODE_PCG) {
                T d = T(0);
#pragma unroll
                for (int q = 0; q < 10 * DPN; ++q) d += xe[q] * ye[q];
                dot += (double)d;
            }
#pragma unroll
            for (int l = 0; l < 10; ++l)
#pragma unroll
                for (int c = 0; c < DPN; ++c) SC::add(ys, M, li[l] * DPN + c, ye[l * DPN + c] * S);
        }
        __syncthreads();
        // 3. flush (node ids: the own range, then the foreign list still in the aux buffer)
        for (int u = threadIdx.x; u < nloc; u += blockDim.x) {
            const uint8_t fl = sfl[u];
            if (HALO) {  // own nodes stored, foreign ones to their halo slots (DPN values each)
                if (DPN == 1) {  // kept apart: the general form costs the FP32 thermal kernel 9 registers
                    const T v = SC::take(ys, M, patch_slot(u)) * invS;
                    if (fl & 1) continue;
                    if (u < nown) a.y[o0 + u] = v;
                    else a.halo[HG ? __ldg(pv.fslot + pm.fa + (u - nown)) : sfsl[u - nown]] = v;
                    continue;
                }
                const int64_t base = u < nown ? (int64_t)(o0 + u) * DPN
                                              : (int64_t)(HG ? __ldg(pv.fslot + pm.fa + (u - nown)) : sfsl[u - nown]) * DPN;
                T* dst = u < nown ? a.y : a.halo;
#pragma unroll
                for (int c = 0; c < DPN; ++c) {
                    const T v = SC::take(ys, M, patch_slot(u) * DPN + c) * invS;
                    if (!((fl >> c) & 1)) dst[base + c] = v;
                }
                continue;
            }
            const int node = u < nown ? o0 + u : sfor[u - nown];
            const bool plain = u < nown && !(fl & kFlagShared);
#pragma unroll
            for (int c = 0; c < DPN; ++c) {
                const T v = SC::take(ys, M, patch_slot(u) * DPN + c) * invS;
                if ((fl >> c) & 1) continue;
                T* dst = a.y + (int64_t)node * DPN + c;
                if (plain) *dst = v;
                else atomicAdd(dst, v);
            }
        }
        // The late shape needs no barrier here: the next gather writes xs and the other
        // flag table, which no flush reads, and the accumulators are zero again.
        if (!LATE) {
            __syncthreads();
            if (NBUF == 1 && threadIdx.x == 0 && has_next) {
                issue_next(patch, k, 0);
                pend |= 1u;
            }
        }
    }
    if (MODE == MODE_PCG) {
        double v[2] = {dot, pdd};
        store_partial<2>(a.part, v);
        if (last_block(&a.st->ticket[TICKET_PATCH])) {
            double t[2];
            grid_total<2>(a.part, gridDim.x, t);
            if (threadIdx.x == 0) {
                PcgState* st = a.st;
                st->ticket[TICKET_PATCH] = 0;
                const double pAp = t[0] + st->cd * t[1];
                st->pAp = pAp;
                if (fabs(pAp) < 1e-30) {  // iterative.rs:85
                    st->flags |= ST_DONE | ST_BREAKDOWN;
                    st->alpha = 0.0;  // no step: the z-form's pending x update adds nothing
                } else {
                    st->alpha = st->rz / pAp;
                }
            }
        }
    }
}

// ------------------------------------------------------------------ node kernels
template <class T>
struct NodeArgs {
    const uint8_t* flags;
    int64_t n;
    int dpn;
    T* x;  // solution (FP64 mode) or FP32 correction xs (mixed)
    T* r;
    T* q;
    const T* dinv;
    T* pbuf0;
    T* pbuf1;
    PcgState* st;
    double* part;
    // mixed refresh
    double* x64;
    double* w64;
    const double* b;
    int vec;  // x, r, q, dinv, pbuf0 and pbuf1 are 16-byte aligned: k_pcg_update uses 16-byte loads
    // halo mode: foreign contributions by slot (dpn values each); node i's slots
    // follow those of nodes < i, hbase[c] = slots of nodes < 32 c, flag bits 3-6 =
    // the node's slot count
    const T* halo;
    const int32_t* hbase;
    const double* halo64;  // mixed refresh: FP64 slots of the FP64 apply (halo mode)
};

// 16-byte vector of T
template <class T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int N = 4;
};
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int N = 2;
};

// x += alpha p, r -= alpha q, z = D^-1 r; r.r and r.z; stopping / refresh decision.
// With aligned vectors (a.vec) every thread streams 16-byte loads of p, q, x, r
// and D^-1, kUnroll vectors in flight, and a scalar loop covers the tail.
// r.r and r.z partials of the node update; the last block sums them, tests
// convergence (FP64) or the refresh criteria (mixed) and sets beta.
template <class T, bool MIXED>
__device__ __forceinline__ void pcg_update_finish(const NodeArgs<T>& a, T acc_rr, T acc_rz) {
    PcgState* st = a.st;
    double v[2] = {(double)acc_rr, (double)acc_rz};
    store_partial<2>(a.part, v);
    if (last_block(&st->ticket[TICKET_UPDATE])) {
        double t[2];
        grid_total<2>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            st->ticket[TICKET_UPDATE] = 0;
            const double rn = sqrt(t[0]);
            if (!MIXED) {
                st->res = rn;
                if (rn < st->tol * st->bnorm || rn < st->abs_tol) {  // iterative.rs:95
                    st->flags |= ST_DONE | ST_CONVERGED;
                    return;
                }
            }
            st->beta = t[1] / st->rz;
            st->rz_old = st->rz;
            st->rz = t[1];
            st->it += 1;
            if (MIXED) {
                st->rmax = fmax(st->rmax, rn);
                const double est = rn * st->s_scale;
                if (est < st->tol * st->bnorm || est < st->abs_tol || rn < st->delta * st->rmax ||
                    st->it >= st->max_it)
                    st->flags |= ST_REFRESH;
            } else if (st->it >= st->max_it) {
                st->flags |= ST_DONE;
            }
        }
    }
}

// k_pcg_update_halo: one 16-byte vector per array in flight per thread, four
// resident blocks (64 registers; the z-form: six, below). The halo loads wait on the slot scan, so warps
// hide that latency better than deeper unrolling: at 128^3 (FP32) 0.095 ms
// against 0.107 ms (two vectors) and 0.20 ms (four, one block per SM).
// The z-form update of the mixed thermal solver streams four vectors instead of
// seven and fits six blocks per SM (42 registers): 0.073 ms at 128^3 against
// 0.085 ms at four blocks and 0.081 ms at eight.
constexpr int kHaloUnroll = 1;
constexpr int kHaloMinBlocks = 4;
constexpr int kHaloMinBlocksZ = 6;
constexpr int kHaloShift = 3;  // flag bits 3-6: halo slots of the node (halo mode)

// ro / dj for the norms of the z-form (FP32: the fast reciprocal-multiply, within
// two units in the last place; the stopping and refresh tests do not need more)
__device__ __forceinline__ float fast_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fast_div(double a, double b) { return a / b; }

// Sum of node j's halo slots, starting at slot s (fixed order: slot order).
template <class T>
__device__ __forceinline__ T halo_sum(const T* __restrict__ halo, int64_t s, int cnt) {
    T h = T(0);
    for (int i = 0; i < cnt; ++i) h += halo[s + i];
    return h;
}

// Node update of a one-DOF operator in halo mode: as the loops of k_pcg_update,
// with q_j = (own-patch sum, stored by the patch kernel) + (node j's halo slots).
// Lane l of a warp takes vector iv (V nodes); the warp's 32 vectors are 32 V
// consecutive nodes starting at a multiple of 32, so its first slot is
// hbase[first / 32] and each lane's first slot follows from a warp scan of the
// lanes' slot counts. Loop conditions are warp-uniform (lanes past the end load
// nothing and count 0 slots).
template <class T, int kU, bool ZF>
__device__ __forceinline__ void pcg_update_halo(const NodeArgs<T>& a, T alpha, T cd, const T* __restrict__ p,
                                                T& acc_rr, T& acc_rz) {
    using VT = typename Vec16<T>::type;
    constexpr int V = Vec16<T>::N;
    const uint8_t* __restrict__ flags = a.flags;
    const T* __restrict__ dinv = a.dinv;
    const T* __restrict__ halo = a.halo;
    T* __restrict__ x = a.x;
    T* __restrict__ r = a.r;
    const T* __restrict__ q = a.q;
    const int lane = threadIdx.x & 31;
    const int64_t n = a.n, nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // ZF (mixed solver's z-form, see k_patch): r holds z = D^-1 r, x is not touched
    // (the next patch kernel updates it) and p is read only where a Dirichlet row needs it
    auto entry = [&](T pj, T qj, T xj, T rj, T dj, uint8_t f, T& xo, T& ro) {
        const T qq = (f & 1) ? cd * pj : qj;
        if (ZF) {
            ro = rj - alpha * (dj * qq);
            const T rr = fast_div(ro, dj);
            acc_rr += rr * rr;
            acc_rz += rr * ro;
            xo = xj;
            return;
        }
        xo = xj + alpha * pj;
        ro = rj - alpha * qq;
        acc_rr += ro * ro;
        acc_rz += ro * (ro * dj);
    };
    // first slot of this lane's V nodes; every lane of the warp calls it
    auto lane_slot = [&](int64_t iv, int tot) {
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int64_t first = __shfl_sync(0xffffffffu, iv, 0) * V;
        return (int64_t)a.hbase[first / 32] + (incl - tot);
    };
    const int64_t nv = a.vec ? n / V : 0;
    int64_t iv = tid;
    for (; iv - lane + 31 + (kU - 1) * nth < nv; iv += kU * nth) {  // all lanes, all u in range
        VT pv[kU] = {}, qv[kU], xv[kU], rv[kU], dv[kU];
        uint8_t fl[kU][V];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int64_t k = iv + u * nth;
            qv[u] = reinterpret_cast<const VT*>(q)[k];
            if (!ZF) xv[u] = reinterpret_cast<const VT*>(x)[k];
            rv[u] = reinterpret_cast<const VT*>(r)[k];
            dv[u] = reinterpret_cast<const VT*>(dinv)[k];
            uint8_t any_dir = 0;
#pragma unroll
            for (int e = 0; e < V; ++e) {
                fl[u][e] = flags[k * V + e];
                any_dir |= fl[u][e];
            }
            if (!ZF || (any_dir & 1)) pv[u] = reinterpret_cast<const VT*>(p)[k];
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int64_t k = iv + u * nth;
            int cnt[V], tot = 0;
#pragma unroll
            for (int e = 0; e < V; ++e) {
                cnt[e] = (fl[u][e] >> kHaloShift) & 15;
                tot += cnt[e];
            }
            int64_t sl = lane_slot(k, tot);
            const T* pe = reinterpret_cast<const T*>(&pv[u]);
            const T* qe = reinterpret_cast<const T*>(&qv[u]);
            const T* xe = reinterpret_cast<const T*>(&xv[u]);
            const T* re = reinterpret_cast<const T*>(&rv[u]);
            const T* de = reinterpret_cast<const T*>(&dv[u]);
            VT xo, ro;
            T* xoe = reinterpret_cast<T*>(&xo);
            T* roe = reinterpret_cast<T*>(&ro);
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const T qj = qe[e] + halo_sum(halo, sl, cnt[e]);
                sl += cnt[e];
                entry(pe[e], qj, xe[e], re[e], de[e], fl[u][e], xoe[e], roe[e]);
            }
            if (!ZF) reinterpret_cast<VT*>(x)[k] = xo;
            reinterpret_cast<VT*>(r)[k] = ro;
        }
    }
    for (; iv - lane < nv; iv += nth) {  // warp-uniform: some lanes may be past nv
        const bool in = iv < nv;
        uint8_t fl[V];
        int cnt[V], tot = 0;
#pragma unroll
        for (int e = 0; e < V; ++e) {
            fl[e] = in ? flags[iv * V + e] : (uint8_t)0;
            cnt[e] = (fl[e] >> kHaloShift) & 15;
            tot += cnt[e];
        }
        int64_t sl = lane_slot(iv, tot);
        if (in) {
            const VT pv = reinterpret_cast<const VT*>(p)[iv], qv = reinterpret_cast<const VT*>(q)[iv];
            const VT xv = ZF ? VT{} : reinterpret_cast<const VT*>(x)[iv], rv = reinterpret_cast<const VT*>(r)[iv];
            const VT dv = reinterpret_cast<const VT*>(dinv)[iv];
            VT xo, ro;
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const T qj = reinterpret_cast<const T*>(&qv)[e] + halo_sum(halo, sl, cnt[e]);
                sl += cnt[e];
                entry(reinterpret_cast<const T*>(&pv)[e], qj, reinterpret_cast<const T*>(&xv)[e],
                      reinterpret_cast<const T*>(&rv)[e], reinterpret_cast<const T*>(&dv)[e], fl[e],
                      reinterpret_cast<T*>(&xo)[e], reinterpret_cast<T*>(&ro)[e]);
            }
            if (!ZF) reinterpret_cast<VT*>(x)[iv] = xo;
            reinterpret_cast<VT*>(r)[iv] = ro;
        }
    }
    // the last n mod V nodes (all nodes when the vectors are not 16-byte aligned):
    // the slot base from the 32-node chunk start
    for (int64_t j = nv * V + tid; j < n; j += nth) {
        const uint8_t f = flags[j];
        int64_t sl = a.hbase[j / 32];
        for (int64_t i = j & ~(int64_t)31; i < j; ++i) sl += (flags[i] >> kHaloShift) & 15;
        T xo, ro;
        entry(p[j], q[j] + halo_sum(halo, sl, (f >> kHaloShift) & 15), ZF ? T(0) : x[j], r[j], dinv[j], f, xo, ro);
        if (!ZF) x[j] = xo;
        r[j] = ro;
    }
}

template <class T, int DPN, bool MIXED>
__global__ void __launch_bounds__(kNodeBS) k_pcg_update(NodeArgs<T> a) {
    PcgState* st = a.st;
    if (st->flags & (ST_DONE | ST_REFRESH)) return;
    const T alpha = (T)st->alpha;
    const T cd = (T)st->cd;
    const T* __restrict__ p = (st->it & 1) ? a.pbuf0 : a.pbuf1;
    const uint8_t* __restrict__ flags = a.flags;
    const T* __restrict__ dinv = a.dinv;
    T* __restrict__ x = a.x;
    T* __restrict__ r = a.r;
    T* __restrict__ q = a.q;
    using VT = typename Vec16<T>::type;
    constexpr int V = Vec16<T>::N;
    const int64_t n = a.n, nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    T acc_rr = T(0), acc_rz = T(0);
    // z-form (the mixed solver, see k_patch): r holds z = D^-1 r and x is updated by the
    // next patch kernel
    constexpr bool ZF = MIXED && std::is_same<T, float>::value;
    // one entry: new x and r (z-form: new z), q zeroed where another patch accumulates into it next time
    auto entry = [&](int64_t j, T pj, T qj, T xj, T rj, T dj, T& xo, T& ro) {
        const uint8_t f = flags[j / DPN];
        const bool dir = (f >> (j % DPN)) & 1;
        const T qq = dir ? cd * pj : qj;
        if (!dir && (f & kFlagShared)) q[j] = T(0);
        if (ZF) {
            ro = rj - alpha * (dj * qq);
            const T rr = fast_div(ro, dj);
            acc_rr += rr * rr;
            acc_rz += rr * ro;
            xo = xj;
            return;
        }
        xo = xj + alpha * pj;
        ro = rj - alpha * qq;
        acc_rr += ro * ro;
        acc_rz += ro * (ro * dj);
    };
    const int64_t nv = a.vec ? n / V : 0;
    int64_t iv = tid;
    for (; iv + (kUnroll - 1) * nth < nv; iv += kUnroll * nth) {
        VT pv[kUnroll], qv[kUnroll], xv[kUnroll], rv[kUnroll], dv[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int64_t k = iv + u * nth;
            pv[u] = reinterpret_cast<const VT*>(p)[k];
            qv[u] = reinterpret_cast<const VT*>(q)[k];
            if (!ZF) xv[u] = reinterpret_cast<const VT*>(x)[k];
            rv[u] = reinterpret_cast<const VT*>(r)[k];
            dv[u] = reinterpret_cast<const VT*>(dinv)[k];
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int64_t k = iv + u * nth;
            const T* pe = reinterpret_cast<const T*>(&pv[u]);
            const T* qe = reinterpret_cast<const T*>(&qv[u]);
            const T* xe = reinterpret_cast<const T*>(&xv[u]);
            const T* re = reinterpret_cast<const T*>(&rv[u]);
            const T* de = reinterpret_cast<const T*>(&dv[u]);
            VT xo, ro;
            T* xoe = reinterpret_cast<T*>(&xo);
            T* roe = reinterpret_cast<T*>(&ro);
#pragma unroll
            for (int e = 0; e < V; ++e) entry(k * V + e, pe[e], qe[e], xe[e], re[e], de[e], xoe[e], roe[e]);
            if (!ZF) reinterpret_cast<VT*>(x)[k] = xo;
            reinterpret_cast<VT*>(r)[k] = ro;
        }
    }
    for (; iv < nv; iv += nth) {
        const VT pv = reinterpret_cast<const VT*>(p)[iv], qv = reinterpret_cast<const VT*>(q)[iv];
        const VT xv = ZF ? VT{} : reinterpret_cast<const VT*>(x)[iv], rv = reinterpret_cast<const VT*>(r)[iv];
        const VT dv = reinterpret_cast<const VT*>(dinv)[iv];
        VT xo, ro;
#pragma unroll
        for (int e = 0; e < V; ++e)
            entry(iv * V + e, reinterpret_cast<const T*>(&pv)[e], reinterpret_cast<const T*>(&qv)[e],
                  reinterpret_cast<const T*>(&xv)[e], reinterpret_cast<const T*>(&rv)[e],
                  reinterpret_cast<const T*>(&dv)[e], reinterpret_cast<T*>(&xo)[e], reinterpret_cast<T*>(&ro)[e]);
        if (!ZF) reinterpret_cast<VT*>(x)[iv] = xo;
        reinterpret_cast<VT*>(r)[iv] = ro;
    }
    for (int64_t j = nv * V + tid; j < n; j += nth) {
        T xo, ro;
        entry(j, p[j], q[j], ZF ? T(0) : x[j], r[j], dinv[j], xo, ro);
        if (!ZF) x[j] = xo;
        r[j] = ro;
    }
    pcg_update_finish<T, MIXED>(a, acc_rr, acc_rz);
}

// Node update of a three-DOF operator in halo mode: one node per lane, its three
// interleaved DOFs of every vector by scalar loads (issued before the slot scan),
// then its slots' three components. A warp's 32 lanes are 32 consecutive nodes
// starting at a multiple of 32, as in pcg_update_halo.
template <class T, bool ZF>
__device__ __forceinline__ void pcg_update_halo3(const NodeArgs<T>& a, T alpha, T cd, const T* __restrict__ p,
                                                 T& acc_rr, T& acc_rz) {
    const uint8_t* __restrict__ flags = a.flags;
    const T* __restrict__ dinv = a.dinv;
    const T* __restrict__ halo = a.halo;
    T* __restrict__ x = a.x;
    T* __restrict__ r = a.r;
    const T* __restrict__ q = a.q;
    const int lane = threadIdx.x & 31;
    const int64_t nn = a.n / 3, nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if constexpr (std::is_same_v<T, float>) {
        if (a.vec) {
            // FP32: two consecutive nodes per lane, so that each vector's six values are
            // three 8-byte loads (a lane's pair starts at DOF 6 m); a warp covers 64
            // nodes starting at a multiple of 64
            const int64_t np2 = nn / 2;
            for (int64_t m = tid; m - lane < np2; m += nth) {
                const bool in = m < np2;
                float pv[6], qv[6], xv[6], rv[6], dv[6];
                uint8_t f[2] = {0, 0};
                if (in) {
                    f[0] = flags[2 * m];
                    f[1] = flags[2 * m + 1];
                    // z-form: p only where a Dirichlet row needs it, x not touched
                    const bool need_p = !ZF || ((f[0] | f[1]) & 7);
    #pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float2 tp = need_p ? reinterpret_cast<const float2*>(p)[3 * m + k] : make_float2(0.f, 0.f);
                        const float2 tq = reinterpret_cast<const float2*>(q)[3 * m + k];
                        const float2 tx = ZF ? make_float2(0.f, 0.f) : reinterpret_cast<const float2*>(x)[3 * m + k];
                        const float2 tr = reinterpret_cast<const float2*>(r)[3 * m + k];
                        const float2 td = reinterpret_cast<const float2*>(dinv)[3 * m + k];
                        pv[2 * k] = tp.x, pv[2 * k + 1] = tp.y;
                        qv[2 * k] = tq.x, qv[2 * k + 1] = tq.y;
                        xv[2 * k] = tx.x, xv[2 * k + 1] = tx.y;
                        rv[2 * k] = tr.x, rv[2 * k + 1] = tr.y;
                        dv[2 * k] = td.x, dv[2 * k + 1] = td.y;
                    }
                }
                const int c0 = (f[0] >> kHaloShift) & 15, c1 = (f[1] >> kHaloShift) & 15;
                const int tot = c0 + c1;
                int incl = tot;
    #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int64_t first = __shfl_sync(0xffffffffu, m, 0) * 2;
                const int64_t s0 = (int64_t)a.hbase[first / 32] + (incl - tot);
                if (!in) continue;
    #pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int cnt = e ? c1 : c0;
                    const int64_t se = s0 + (e ? c0 : 0);
    #pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int v = 3 * e + c;
                        float h = 0.0f;
                        for (int i = 0; i < cnt; ++i) h += halo[3 * (se + i) + c];
                        const float qq = ((f[e] >> c) & 1) ? (float)cd * pv[v] : qv[v] + h;
                        if (ZF) {  // rv holds z = D^-1 r
                            rv[v] = rv[v] - (float)alpha * (dv[v] * qq);
                            const float rr = fast_div(rv[v], dv[v]);
                            acc_rr += rr * rr;
                            acc_rz += rr * rv[v];
                            continue;
                        }
                        xv[v] = xv[v] + (float)alpha * pv[v];
                        rv[v] = rv[v] - (float)alpha * qq;
                        acc_rr += rv[v] * rv[v];
                        acc_rz += rv[v] * (rv[v] * dv[v]);
                    }
                }
    #pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (!ZF) reinterpret_cast<float2*>(x)[3 * m + k] = make_float2(xv[2 * k], xv[2 * k + 1]);
                    reinterpret_cast<float2*>(r)[3 * m + k] = make_float2(rv[2 * k], rv[2 * k + 1]);
                }
            }
            // an odd last node: its first slot from the 32-node chunk start
            for (int64_t nd = 2 * np2 + tid; nd < nn; nd += nth) {
                const uint8_t f = flags[nd];
                const int cnt = (f >> kHaloShift) & 15;
                int64_t s0 = a.hbase[nd / 32];
                for (int64_t i = nd & ~(int64_t)31; i < nd; ++i) s0 += (flags[i] >> kHaloShift) & 15;
    #pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t j = 3 * nd + c;
                    T h = T(0);
                    for (int i = 0; i < cnt; ++i) h += halo[3 * (s0 + i) + c];
                    const T qq = ((f >> c) & 1) ? cd * p[j] : q[j] + h;
                    if (ZF) {
                        const T zo = r[j] - alpha * (dinv[j] * qq);
                        const T rr = fast_div(zo, dinv[j]);
                        r[j] = zo;
                        acc_rr += rr * rr;
                        acc_rz += rr * zo;
                        continue;
                    }
                    const T xo = x[j] + alpha * p[j];
                    const T ro = r[j] - alpha * qq;
                    x[j] = xo;
                    r[j] = ro;
                    acc_rr += ro * ro;
                    acc_rz += ro * (ro * dinv[j]);
                }
            }
            return;
        }
    }
    for (int64_t nd = tid; nd - lane < nn; nd += nth) {
        const bool in = nd < nn;
        T pv[3], qv[3], xv[3], rv[3], dv[3];
        uint8_t f = 0;
        if (in) {
            f = flags[nd];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int64_t j = 3 * nd + c;
                pv[c] = p[j];
                qv[c] = q[j];
                xv[c] = ZF ? T(0) : x[j];
                rv[c] = r[j];
                dv[c] = dinv[j];
            }
        }
        const int cnt = (f >> kHaloShift) & 15;
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int64_t first = __shfl_sync(0xffffffffu, nd, 0);
        const int64_t s0 = (int64_t)a.hbase[first / 32] + (incl - cnt);
        if (!in) continue;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T h = T(0);
            for (int i = 0; i < cnt; ++i) h += halo[3 * (s0 + i) + c];
            const T qq = ((f >> c) & 1) ? cd * pv[c] : qv[c] + h;
            if (ZF) {
                const T zo = rv[c] - alpha * (dv[c] * qq);
                const T rr = fast_div(zo, dv[c]);
                r[3 * nd + c] = zo;
                acc_rr += rr * rr;
                acc_rz += rr * zo;
                continue;
            }
            const T xo = xv[c] + alpha * pv[c];
            const T ro = rv[c] - alpha * qq;
            x[3 * nd + c] = xo;
            r[3 * nd + c] = ro;
            acc_rr += ro * ro;
            acc_rz += ro * (ro * dv[c]);
        }
    }
}

// Node update of a PCG in halo mode (see pcg_update_halo / pcg_update_halo3).
template <class T, int DPN, bool MIXED>
__global__ void __launch_bounds__(kNodeBS, (MIXED && DPN == 1 && std::is_same<T, float>::value) ? kHaloMinBlocksZ
                                                                                             : kHaloMinBlocks)
    k_pcg_update_halo(NodeArgs<T> a) {
    PcgState* st = a.st;
    if (st->flags & (ST_DONE | ST_REFRESH)) return;
    const T* __restrict__ p = (st->it & 1) ? a.pbuf0 : a.pbuf1;
    T acc_rr = T(0), acc_rz = T(0);
    if (DPN == 1)
        pcg_update_halo<T, kHaloUnroll, MIXED && std::is_same<T, float>::value>(a, (T)st->alpha, (T)st->cd, p,
                                                                                 acc_rr, acc_rz);
    else pcg_update_halo3<T, MIXED && std::is_same<T, float>::value>(a, (T)st->alpha, (T)st->cd, p, acc_rr, acc_rz);
    pcg_update_finish<T, MIXED>(a, acc_rr, acc_rz);
}

// FP64 mode start: x = 0, r = b, p_old = 0, q = 0; ||b||, r.z.
template <class T>
__global__ void __launch_bounds__(kNodeBS) k_pcg_init(NodeArgs<T> a) {
    const int64_t n = a.n, nth = (int64_t)gridDim.x * blockDim.x;
    double bb = 0.0, rz = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += nth) {
        const double bi = a.b[i];
        a.x[i] = T(0);
        a.r[i] = (T)bi;
        a.q[i] = T(0);
        a.pbuf0[i] = T(0);
        bb += bi * bi;
        rz += bi * (bi * (double)a.dinv[i]);
    }
    double v[2] = {bb, rz};
    store_partial<2>(a.part, v);
    if (last_block(&a.st->ticket[TICKET_AUX])) {
        double t[2];
        grid_total<2>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            PcgState* st = a.st;
            st->ticket[TICKET_AUX] = 0;
            st->bnorm = sqrt(t[0]);
            st->res = st->bnorm;
            st->rz = t[1];
            st->beta = 0.0;
            st->it = 0;
            st->nupd = 0;
            st->s_scale = 1.0;
            st->rmax = 1.0;
            if (st->bnorm < 1e-25) {  // iterative.rs:60-68
                st->flags |= ST_DONE | ST_CONVERGED;
                st->res = 0.0;
            }
            if (st->max_it <= 0) st->flags |= ST_DONE;
        }
    }
}

// MIXED start, pass 1: x64 = 0, xs = 0, q = 0, w64 = 0, p_old = 0; ||b||.
__global__ void __launch_bounds__(kNodeBS) k_mixed_init1(NodeArgs<float> a) {
    const int64_t n = a.n, nth = (int64_t)gridDim.x * blockDim.x;
    double bb = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += nth) {
        const double bi = a.b[i];
        a.x64[i] = 0.0;
        a.w64[i] = 0.0;
        a.x[i] = 0.0f;
        a.q[i] = 0.0f;
        a.pbuf0[i] = 0.0f;
        bb += bi * bi;
    }
    double v[1] = {bb};
    store_partial<1>(a.part, v);
    if (last_block(&a.st->ticket[TICKET_AUX])) {
        double t[1];
        grid_total<1>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            PcgState* st = a.st;
            st->ticket[TICKET_AUX] = 0;
            st->bnorm = sqrt(t[0]);
            st->res = st->bnorm;
            st->s_scale = st->bnorm;
            st->beta = 0.0;
            st->it = 0;
            st->nupd = 0;
            st->rmax = 1.0;
            if (st->bnorm < 1e-25) {
                st->flags |= ST_DONE | ST_CONVERGED;
                st->res = 0.0;
            }
            if (st->max_it <= 0) st->flags |= ST_DONE;
        }
    }
}

// MIXED start, pass 2: r = b / ||b|| (FP32), r.z.
__global__ void __launch_bounds__(kNodeBS) k_mixed_init2(NodeArgs<float> a) {
    if (a.st->flags & ST_DONE) return;
    const int64_t n = a.n, nth = (int64_t)gridDim.x * blockDim.x;
    const double inv = 1.0 / a.st->s_scale;
    double rz = 0.0;
    const bool zf = true;  // the mixed solver keeps z = D^-1 r (see k_patch)
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += nth) {
        const float ri = (float)(a.b[i] * inv);
        const float zi = ri * a.dinv[i];
        a.r[i] = zf ? zi : ri;
        rz += (double)(ri * zi);
    }
    double v[1] = {rz};
    store_partial<1>(a.part, v);
    if (last_block(&a.st->ticket[TICKET_AUX])) {
        double t[1];
        grid_total<1>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            a.st->ticket[TICKET_AUX] = 0;
            a.st->rz = t[0];
        }
    }
}

// MIXED refresh 1: x64 += s xs, xs = 0. In the z-form xs still
// lacks the last step alpha p of the iteration that asked for the refresh (the next
// patch kernel would have added it): it is added here, and k_refresh_residual sets
// alpha to 0 so that no later patch kernel adds it again.
__global__ void __launch_bounds__(kNodeBS) k_refresh_flush(NodeArgs<float> a) {
    const double s = a.st->s_scale;
    const bool zf = true;  // z-form (see k_patch)
    const float alpha = zf ? (float)a.st->alpha : 0.0f;
    const float* p = (a.st->it & 1) ? a.pbuf1 : a.pbuf0;  // the last direction
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        const float xi = zf ? a.x[i] + alpha * p[i] : a.x[i];
        a.x64[i] += s * (double)xi;
        a.x[i] = 0.0f;
    }
}

// MIXED refresh 3: w = b - K_bc x64 (w holds K x64 on free rows); ||w|| decides
// convergence (FP64 true residual).
__global__ void __launch_bounds__(kNodeBS) k_refresh_residual(NodeArgs<float> a) {
    PcgState* st = a.st;
    const double cd = st->cd;
    double rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool dir = (a.flags[i / a.dpn] >> (i % a.dpn)) & 1;
        const double kx = dir ? cd * a.x64[i] : a.w64[i];
        const double ri = a.b[i] - kx;
        a.w64[i] = ri;
        rr += ri * ri;
    }
    double v[1] = {rr};
    store_partial<1>(a.part, v);
    if (last_block(&st->ticket[TICKET_AUX])) {
        double t[1];
        grid_total<1>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            st->ticket[TICKET_AUX] = 0;
            const double s_new = sqrt(t[0]);
            st->alpha = 0.0;  // the last step is in x64 now (k_refresh_flush)
            st->nupd += 1;
            st->res = s_new;
            st->s_new = s_new;
            if (s_new < st->tol * st->bnorm || s_new < st->abs_tol) {
                st->flags = (st->flags & ~ST_REFRESH) | ST_DONE | ST_CONVERGED;
            } else {
                st->ratio = st->s_scale / s_new;
            }
        }
    }
}

// Sum over the warp of lanes' slot counts before this lane: the exclusive prefix
// that, added to hbase[node / 32], gives the node's first halo slot. Every lane of
// the warp calls it; the warp's lanes hold 32 consecutive nodes from a multiple of
// 32 (lanes past the end pass cnt = 0).
__device__ __forceinline__ int halo_prefix(int cnt, int lane) {
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    return incl - cnt;
}

// MIXED refresh 3, halo mode: as k_refresh_residual, with K x64 on free rows =
// (own-patch sum in w) + (the node's FP64 halo slots, in slot order). Threads
// take nodes; the grid is a multiple of 32 threads, so warps cover aligned
// 32-node chunks and the loop condition is warp-uniform.
__global__ void __launch_bounds__(kNodeBS) k_refresh_residual_halo(NodeArgs<float> a) {
    PcgState* st = a.st;
    const double cd = st->cd;
    const int dpn = a.dpn, lane = threadIdx.x & 31;
    const int64_t nn = a.n / dpn, nth = (int64_t)gridDim.x * blockDim.x;
    double rr = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j - lane < nn; j += nth) {
        const bool in = j < nn;
        const uint8_t f = in ? a.flags[j] : (uint8_t)0;
        const int cnt = (f >> kHaloShift) & 15;
        const int pre = halo_prefix(cnt, lane);
        if (!in) continue;
        const int64_t s0 = (int64_t)a.hbase[j >> 5] + pre;
        for (int c = 0; c < dpn; ++c) {
            const int64_t i = j * dpn + c;
            double kx;
            if ((f >> c) & 1) {
                kx = cd * a.x64[i];
            } else {
                kx = a.w64[i];
                for (int k = 0; k < cnt; ++k) kx += a.halo64[(s0 + k) * dpn + c];
            }
            const double ri = a.b[i] - kx;
            a.w64[i] = ri;
            rr += ri * ri;
        }
    }
    double v[1] = {rr};
    store_partial<1>(a.part, v);
    if (last_block(&st->ticket[TICKET_AUX])) {
        double t[1];
        grid_total<1>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            st->ticket[TICKET_AUX] = 0;
            const double s_new = sqrt(t[0]);
            st->alpha = 0.0;  // the last step is in x64 now (k_refresh_flush)
            st->nupd += 1;
            st->res = s_new;
            st->s_new = s_new;
            if (s_new < st->tol * st->bnorm || s_new < st->abs_tol) {
                st->flags = (st->flags & ~ST_REFRESH) | ST_DONE | ST_CONVERGED;
            } else {
                st->ratio = st->s_scale / s_new;
            }
        }
    }
}

// After a FREE or LIFT pass in halo mode: y_j += node j's halo slots (slot order)
// on free rows; with `dir_rows`, Dirichlet rows y = cd x (as k_dir_rows). Node-
// per-thread with warp-aligned 32-node chunks (grid a multiple of 32 threads).
template <class T>
__global__ void __launch_bounds__(kNodeBS) k_halo_combine(const uint8_t* __restrict__ flags,
                                                          const int32_t* __restrict__ hbase,
                                                          const T* __restrict__ halo, int dpn, int64_t nn,
                                                          double cd, const T* __restrict__ x, T* __restrict__ y,
                                                          int dir_rows) {
    const int lane = threadIdx.x & 31;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j - lane < nn; j += nth) {
        const bool in = j < nn;
        const uint8_t f = in ? flags[j] : (uint8_t)0;
        const int cnt = (f >> kHaloShift) & 15;
        const int pre = halo_prefix(cnt, lane);
        if (!in) continue;
        const int64_t s0 = (int64_t)hbase[j >> 5] + pre;
        for (int c = 0; c < dpn; ++c) {
            const int64_t i = j * dpn + c;
            if ((f >> c) & 1) {
                if (dir_rows) y[i] = (T)(cd * (double)x[i]);
                continue;
            }
            if (cnt == 0) continue;
            T h = y[i];
            for (int k = 0; k < cnt; ++k) h += halo[(s0 + k) * dpn + c];
            y[i] = h;
        }
    }
}

// MIXED refresh 4: r = w / ||w||, current p rescaled, r.z recomputed.
__global__ void __launch_bounds__(kNodeBS) k_refresh_rescale(NodeArgs<float> a) {
    PcgState* st = a.st;
    if (st->flags & ST_DONE) return;
    const double inv = 1.0 / st->s_new;
    const float ratio = (float)st->ratio;
    const bool zf = true;  // z-form: r holds z = D^-1 r
    float* p = (st->it & 1) ? a.pbuf1 : a.pbuf0;  // direction the next apply reads
    double rz = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t fl = a.flags[i / a.dpn];
        const double wi = a.w64[i];
        if (!((fl >> (i % a.dpn)) & 1) && (fl & kFlagShared)) a.w64[i] = 0.0;
        const float ri = (float)(wi * inv);
        const float zi = ri * a.dinv[i];
        a.r[i] = zf ? zi : ri;
        p[i] *= ratio;
        rz += (double)(ri * zi);
    }
    double v[1] = {rz};
    store_partial<1>(a.part, v);
    if (last_block(&st->ticket[TICKET_AUX])) {
        double t[1];
        grid_total<1>(a.part, gridDim.x, t);
        if (threadIdx.x == 0) {
            st->ticket[TICKET_AUX] = 0;
            const double ratio2 = st->ratio * st->ratio;
            st->beta = t[0] / (st->rz_old * ratio2);
            st->rz = t[0];
            st->s_scale = st->s_new;
            st->rmax = 1.0;
            st->flags &= ~ST_REFRESH;
            if (st->it >= st->max_it) st->flags |= ST_DONE;
        }
    }
}

// y_D = cd x_D after a MODE_FREE pass
template <class T>
__global__ void k_dir_rows(const uint8_t* flags, int dpn, int64_t n, double cd, const T* x, T* y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if ((flags[i / dpn] >> (i % dpn)) & 1) y[i] = (T)(cd * (double)x[i]);
}

}  // namespace geo
