// FP32 thermal patch kernel of the mixed-precision PCG (PCG mode, affine
// elements, own-node slices by bulk copy): the same operation and the same
// shared-memory pipeline as k_patch<ThermalK<float, 1>, float, MODE_PCG> in
// mf_kernels.cuh, written for the instruction budget of the solver's dominant
// launch. Differences:
//   * each thread applies K_e to two elements at once in packed FP32x2
//     arithmetic (sm_100 FFMA2 / FADD2 / FMUL2), so the element arithmetic
//     issues half the instructions;
//   * the fixed-point scale S of the patch is folded into the element's G
//     (6 multiplies instead of 10), and 1/S is formed exactly from S's exponent;
//   * the patch's own nodes, one contiguous id range, are gathered and flushed
//     four at a time: 16-byte shared loads of the bulk-copied D^-1, r, p_old
//     slices and flags, 16-byte stores of p, of the node table and of q. The
//     node tables are addressed through a per-patch base shifted by o0 mod 4,
//     so that every group of four consecutive own nodes is 16-byte aligned in
//     shared memory as in global memory; groups that straddle the ends of the
//     own range fall back to per-node stores.
// Foreign nodes, the halo slots, the mbarrier pipeline, the bounded waits and
// the deterministic reductions are those of the general kernel.
#pragma once

#include "mf_kernels.cuh"

namespace geo {

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, exactly (b * -1 + a is a single rounding)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }

// y = K_e x for two elements (.x and .y), G already scaled: the scalar form of
// ThermalK<float, 1>::apply (matfree.cuh) on packed pairs. Outputs are
// accumulated as soon as their quadrature-point terms exist, to keep few pairs live.
__device__ __forceinline__ void thermal_apply_pair(const float2 (&G)[6], const float2 (&x)[10], float2 (&y)[10]) {
    const float2 B4 = f2((float)(4.0 * kQb)), D4 = f2((float)(4.0 * (kQa - kQb))),
                 B4m1 = f2((float)(4.0 * kQb - 1.0));
    float2 base[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float2 s = x[m];
#pragma unroll
        for (int n = 0; n < 4; ++n)
            if (n != m) s = add2(s, x[edge_of(m, n)]);
        base[m] = sub2(mul2(B4, s), x[m]);
    }
    float2 Phi[4];
#pragma unroll
    for (int k = 0; k < 6; ++k) y[4 + k] = f2(0.0f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float2 h[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) h[m] = fma2(D4, m == q ? x[m] : x[edge_of(m, q)], base[m]);
        const float2 g0 = sub2(h[1], h[0]), g1 = sub2(h[2], h[0]), g2 = sub2(h[3], h[0]);
        const float2 v0 = fma2(G[2], g2, fma2(G[1], g1, mul2(G[0], g0)));
        const float2 v1 = fma2(G[4], g2, fma2(G[3], g1, mul2(G[1], g0)));
        const float2 v2 = fma2(G[5], g2, fma2(G[4], g1, mul2(G[2], g0)));
        const float2 phi[4] = {sub2(f2(0.0f), add2(add2(v0, v1), v2)), v0, v1, v2};
#pragma unroll
        for (int m = 0; m < 4; ++m) Phi[m] = q == 0 ? phi[m] : add2(Phi[m], phi[m]);
        // y_q gets D4 phi_{q,q}; edge (q, m) gets D4 phi_{q,m}
        y[q] = mul2(D4, phi[q]);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int m = edge_v(k, 0), n = edge_v(k, 1);
            if (q == m) y[4 + k] = fma2(D4, phi[n], y[4 + k]);
            if (q == n) y[4 + k] = fma2(D4, phi[m], y[4 + k]);
        }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) y[m] = fma2(B4m1, Phi[m], y[m]);
#pragma unroll
    for (int k = 0; k < 6; ++k) y[4 + k] = fma2(B4, add2(Phi[edge_v(k, 0)], Phi[edge_v(k, 1)]), y[4 + k]);
}

// Node tables of the patch kernel: xs (FP32 node values) and ys (INT32 fixed-point
// accumulators), each max_local + 4 entries from a 16-byte aligned start, then the
// own-node slices. Offsets from the start of the node-table region.
__host__ __device__ inline uint32_t t32_table_entries(int max_local) { return ((uint32_t)max_local + 4u + 3u) & ~3u; }
__host__ __device__ inline size_t t32_tables_bytes(int max_local, int max_own) {
    return 16 + 2 * (size_t)t32_table_entries(max_local) * 4 + own_bytes<float>(max_own, 1);
}

template <int NBUF, int HG>
__global__ void __launch_bounds__(kPatchBS, 3) k_patch_t32(PatchView pv, const float* __restrict__ qd_all,
                                                             PatchArgs<float> a) {
    using K = ThermalK<float, 1>;
    constexpr uint32_t LCB = patch_bytes_lc<K, float>(), QDB = patch_bytes_qd<K, float>();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // [0..NBUF): element data; [2]: own-node slices
    unsigned char* ebuf = smem + 32;
    unsigned char* abuf = smem + patch_smem_fixed<K, float, NBUF>();
    const int HMODE = HG ? 2 : (pv.halo != 0 ? 1 : 0);
    const uint32_t AUX = patch_aux_bytes(pv.max_for, HMODE), AIDS = patch_aux_ids(pv.max_for);
    const uint32_t AFL = patch_aux_flags(pv.max_for);
    unsigned char* tb = smem + ((patch_smem_tables<K, float, NBUF>(pv.max_for, HMODE) + 15) & ~(size_t)15);
    const uint32_t TE = t32_table_entries(pv.max_local);
    float* xs_al = reinterpret_cast<float*>(tb);
    int* ys_al = reinterpret_cast<int*>(xs_al + TE);
    const uint32_t OCAP = own_cap<float>(pv.max_own, 1);
    float* own_d = reinterpret_cast<float*>(ys_al + TE);
    float* own_r = own_d + OCAP;
    float* own_p = own_r + OCAP;
    uint8_t* own_f = reinterpret_cast<uint8_t*>(own_p + OCAP);
    __shared__ unsigned s_lo[2], s_hi[2];
    if (a.st->flags & (ST_DONE | ST_REFRESH)) return;
    const float beta = (float)a.st->beta;
    const bool odd = a.st->it & 1;
    const float* __restrict__ pold = odd ? a.pbuf1 : a.pbuf0;
    float* __restrict__ pnew = odd ? a.pbuf0 : a.pbuf1;
    const float* __restrict__ rg = a.r;
    const float* __restrict__ dg = a.dinv;
    if (threadIdx.x == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&bar[b], 1);
        mbar_init(&bar[2], 1);
        mbar_fence_init();
        s_lo[0] = s_lo[1] = 0xffffffffu;
        s_hi[0] = s_hi[1] = 0u;
    }
    __syncthreads();
    auto issue = [&](int patch, int b) {
        PatchMeta m;
        m.n_el = pv.pe[patch + 1] - pv.pe[patch];
        m.o0 = pv.po[patch];
        m.nown = pv.po[patch + 1] - m.o0;
        m.nfor = pv.pf[patch + 1] - pv.pf[patch];
        m.fa = pv.pfa[patch];
        m.bound = pv.bound32[patch];
        m.pad0 = m.pad1 = 0;
        unsigned char* ab = abuf + (size_t)b * AUX;
        *reinterpret_cast<PatchMeta*>(ab) = m;
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
    auto issue_own = [&](int patch) {
        const int o0 = pv.po[patch], o1 = pv.po[patch + 1];
        const int a0 = o0 & ~3, nv = ((o1 + 3) & ~3) - a0;
        const int f0 = o0 & ~15, nf = ((o1 + 15) & ~15) - f0;
        const uint32_t vb = (uint32_t)nv * 4u;
        mbar_expect_tx(&bar[2], 3u * vb + (uint32_t)nf);
        if (nv) {
            bulk_g2s(own_d, dg + a0, vb, &bar[2]);
            bulk_g2s(own_r, rg + a0, vb, &bar[2]);
            bulk_g2s(own_p, pold + a0, vb, &bar[2]);
        }
        if (nf) bulk_g2s(own_f, pv.flags + f0, (uint32_t)nf, &bar[2]);
    };
    if (threadIdx.x == 0 && blockIdx.x < pv.n_patches) {
        issue(blockIdx.x, 0);
        issue_own(blockIdx.x);
    }
    uint32_t phase = 0;
    uint32_t pend = blockIdx.x < pv.n_patches ? 5u : 0u;
    double dot = 0.0, pdd = 0.0;
    const int t = threadIdx.x;
    int k = 0;
    for (int patch = blockIdx.x; patch < pv.n_patches; patch += gridDim.x, ++k) {
        const int b = NBUF == 2 ? (k & 1) : 0;
        if (NBUF == 2 && t == 0 && patch + (int)gridDim.x < pv.n_patches) {
            issue(patch + gridDim.x, b ^ 1);
            pend |= 1u << (b ^ 1);
        }
        bool ok = mbar_wait(&bar[b], (phase >> b) & 1);
        if (ok) {
            phase ^= 1u << b;
            pend &= ~(1u << b);
        }
        const bool ok2 = mbar_wait(&bar[2], (phase >> 2) & 1);
        if (ok2) {
            phase ^= 4u;
            pend &= ~4u;
        }
        ok = ok && ok2;
        if (__syncthreads_or(!ok)) {
            if (t == 0) {
                atomicOr(a.err, DEV_ERR_TIMEOUT);
                for (int q = 0; q < 3; ++q)
                    if ((pend >> q) & 1) mbar_wait(&bar[q], (phase >> q) & 1);
            }
            return;
        }
        const unsigned char* ab = abuf + (size_t)b * AUX;
        const PatchMeta pm = *reinterpret_cast<const PatchMeta*>(ab);
        const int* __restrict__ sfor = reinterpret_cast<const int*>(ab + sizeof(PatchMeta));
        const uint8_t* __restrict__ sffl = ab + sizeof(PatchMeta) + AIDS;
        const int* __restrict__ sfsl = reinterpret_cast<const int*>(ab + sizeof(PatchMeta) + AIDS + AFL);
        const int n_el = pm.n_el, o0 = pm.o0, nown = pm.nown, nfor = pm.nfor, o1 = o0 + nown;
        const int sh = o0 & 3, a0 = o0 & ~3;
        float* xsp = xs_al + sh;  // xsp[u]: local node u; 16-byte groups of own nodes
        int* ysp = ys_al + sh;
        float lo = 3.0e38f, hi = -3.0e38f;
        // 1a. own nodes in groups of four (global ids a0 + 4c .. a0 + 4c + 3)
        const int nch = (o1 - a0 + 3) >> 2;
        const float2 bb = f2(beta);
        for (int c = t; c < nch; c += kPatchBS) {
            const float4 d4 = reinterpret_cast<const float4*>(own_d)[c];
            const float4 r4 = reinterpret_cast<const float4*>(own_r)[c];
            const float4 p4 = reinterpret_cast<const float4*>(own_p)[c];
            const uint32_t fw = *reinterpret_cast<const uint32_t*>(own_f + (o0 & 12) + 4 * c);
            const float2 pa = fma2(make_float2(d4.x, d4.y), make_float2(r4.x, r4.y), mul2(bb, make_float2(p4.x, p4.y)));
            const float2 pb = fma2(make_float2(d4.z, d4.w), make_float2(r4.z, r4.w), mul2(bb, make_float2(p4.z, p4.w)));
            const float pn[4] = {pa.x, pa.y, pb.x, pb.y};
            float v[4];
            const int g0 = a0 + 4 * c;
            const bool full = g0 >= o0 && g0 + 4 <= o1;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool in = full || (g0 + j >= o0 && g0 + j < o1);
                const bool dir = (fw >> (8 * j)) & 1u;
                v[j] = dir ? 0.0f : pn[j];
                if (in) {
                    if (dir) pdd += (double)(pn[j] * pn[j]);
                    lo = fminf(lo, v[j]);
                    hi = fmaxf(hi, v[j]);
                }
            }
            if (full) {
                reinterpret_cast<float4*>(pnew)[(g0 >> 2)] = make_float4(pn[0], pn[1], pn[2], pn[3]);
                reinterpret_cast<float4*>(xs_al)[c] = make_float4(v[0], v[1], v[2], v[3]);
                reinterpret_cast<int4*>(ys_al)[c] = make_int4(0, 0, 0, 0);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (g0 + j >= o0 && g0 + j < o1) {
                        pnew[g0 + j] = pn[j];
                        xs_al[4 * c + j] = v[j];
                        ys_al[4 * c + j] = 0;
                    }
            }
        }
        // 1b. foreign nodes (global gather, two in flight per thread)
        for (int f0 = t; f0 < nfor; f0 += 2 * kPatchBS) {
            const int f1 = f0 + kPatchBS;
            const bool has1 = f1 < nfor;
            const int n0 = sfor[f0], n1 = has1 ? sfor[f1] : n0;
            const float d0 = __ldg(dg + n0), r0 = __ldg(rg + n0), q0 = __ldg(pold + n0);
            const float d1 = __ldg(dg + n1), r1 = __ldg(rg + n1), q1 = __ldg(pold + n1);
            const float2 pn = fma2(make_float2(d0, d1), make_float2(r0, r1), mul2(bb, make_float2(q0, q1)));
            const float v0 = (sffl[f0] & 1) ? 0.0f : pn.x;
            xsp[nown + f0] = v0;
            ysp[nown + f0] = 0;
            lo = fminf(lo, v0);
            hi = fmaxf(hi, v0);
            if (has1) {
                const float v1 = (sffl[f1] & 1) ? 0.0f : pn.y;
                xsp[nown + f1] = v1;
                ysp[nown + f1] = 0;
                lo = fminf(lo, v1);
                hi = fmaxf(hi, v1);
            }
        }
        {
            const unsigned l = __reduce_min_sync(0xffffffffu, float_key(lo));
            const unsigned h = __reduce_max_sync(0xffffffffu, float_key(hi));
            if ((t & 31) == 0) {
                atomicMin(&s_lo[k & 1], l);
                atomicMax(&s_hi[k & 1], h);
            }
        }
        __syncthreads();
        if (t == 0 && patch + (int)gridDim.x < pv.n_patches) {
            issue_own(patch + gridDim.x);
            pend |= 4u;
        }
        // 2. scale S (power of two) and its exact inverse, then the elements in pairs
        float S = 1.0f, invS = 1.0f;
        {
            const float l = key_float(s_lo[k & 1]), h = key_float(s_hi[k & 1]);
            if (h >= l) {
                const float half = __fmul_ru(__fsub_ru(h, l), 0.5f);
                const float mabs = fmaxf(fabsf(l), fabsf(h));
                const float bx = __fmul_ru(pm.bound, __fmaf_ru(mabs, 1.52587890625e-05f, half));
                if (bx > 0.0f) {
                    S = pow2_floor(Scatter<float>::kLim / bx);
                    invS = __uint_as_float(0x7f000000u - __float_as_uint(S));  // 2^-e for S = 2^e
                }
            }
            if (t < 1) {
                s_lo[(k + 1) & 1] = 0xffffffffu;
                s_hi[(k + 1) & 1] = 0u;
            }
        }
        const uint32_t* lcs = reinterpret_cast<const uint32_t*>(ebuf + (size_t)b * (LCB + QDB));
        const float* qds = reinterpret_cast<const float*>(ebuf + (size_t)b * (LCB + QDB) + LCB);
        float dpatch = 0.0f;
        if (t < n_el) {
            const int e0 = t, e1 = t + kPatchBS < n_el ? t + kPatchBS : t;  // a lone element: its own pair, once
            const bool two = e1 != e0;
            int li0[10], li1[10];
#pragma unroll
            for (int l2 = 0; l2 < 5; ++l2) {
                const uint32_t w0 = lcs[l2 * kPatchElems + e0], w1 = lcs[l2 * kPatchElems + e1];
                li0[2 * l2] = (int)(w0 & 0xffffu);
                li0[2 * l2 + 1] = (int)(w0 >> 16);
                li1[2 * l2] = (int)(w1 & 0xffffu);
                li1[2 * l2 + 1] = (int)(w1 >> 16);
            }
            float2 G[6], xe[10], ye[10];
            const float2 SS = f2(S);
#pragma unroll
            for (int j = 0; j < 6; ++j) G[j] = mul2(SS, make_float2(qds[j * kPatchElems + e0], qds[j * kPatchElems + e1]));
#pragma unroll
            for (int l = 0; l < 10; ++l) xe[l] = make_float2(xsp[li0[l]], xsp[li1[l]]);
            thermal_apply_pair(G, xe, ye);
            float2 d = mul2(xe[0], ye[0]);
#pragma unroll
            for (int l = 1; l < 10; ++l) d = fma2(xe[l], ye[l], d);
            dpatch = two ? d.x + d.y : d.x;
#pragma unroll
            for (int l = 0; l < 10; ++l) atomicAdd(ysp + li0[l], __float2int_rn(ye[l].x));
            if (two) {
#pragma unroll
                for (int l = 0; l < 10; ++l) atomicAdd(ysp + li1[l], __float2int_rn(ye[l].y));
            }
        }
        dot += (double)dpatch * (double)invS;
        __syncthreads();
        // 3. flush: own nodes in groups of four (q, plain stores), foreign entries to their halo slots
        for (int c = t; c < nch; c += kPatchBS) {
            const int4 y4 = reinterpret_cast<const int4*>(ys_al)[c];
            const float2 ia = mul2(make_float2((float)y4.x, (float)y4.y), f2(invS));
            const float2 ib = mul2(make_float2((float)y4.z, (float)y4.w), f2(invS));
            const int g0 = a0 + 4 * c;
            if (g0 >= o0 && g0 + 4 <= o1) {
                reinterpret_cast<float4*>(a.y)[g0 >> 2] = make_float4(ia.x, ia.y, ib.x, ib.y);
            } else {
                const float v[4] = {ia.x, ia.y, ib.x, ib.y};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (g0 + j >= o0 && g0 + j < o1) a.y[g0 + j] = v[j];
            }
        }
        for (int f = t; f < nfor; f += kPatchBS) {
            if (sffl[f] & 1) continue;
            const int slot = HG ? __ldg(pv.fslot + pm.fa + f) : sfsl[f];
            a.halo[slot] = (float)ysp[nown + f] * invS;
        }
        __syncthreads();
        if (NBUF == 1 && t == 0 && patch + (int)gridDim.x < pv.n_patches) {
            issue(patch + gridDim.x, 0);
            pend |= 1u;
        }
    }
    double v[2] = {dot, pdd};
    store_partial<2>(a.part, v);
    if (last_block(&a.st->ticket[TICKET_PATCH])) {
        double tt[2];
        grid_total<2>(a.part, gridDim.x, tt);
        if (threadIdx.x == 0) {
            PcgState* st = a.st;
            st->ticket[TICKET_PATCH] = 0;
            const double pAp = tt[0] + st->cd * tt[1];
            st->pAp = pAp;
            if (fabs(pAp) < 1e-30) {  // iterative.rs:85
                st->flags |= ST_DONE | ST_BREAKDOWN;
            } else {
                st->alpha = st->rz / pAp;
            }
        }
    }
}

}  // namespace geo
