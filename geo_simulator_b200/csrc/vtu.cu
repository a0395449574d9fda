// VTK output of a device mesh and its fields: the drop-in for VtkWriter::write_vtu
// (mesh/vtk_writer.rs:104-265), VtkWriter::write (legacy .vtk, :13-101) and
// VtkWriter::write_nodal_vtu (:531-789), byte for byte.
//
// The file is ASCII XML in which every coordinate, index and field value is
// printed with Rust's `{}` (decimal.cuh). The text is produced on the GPU from
// the resident mesh and fields, section by section (points, connectivity,
// offsets, types, each field):
//   1. one thread per item (a point line, an element's 10 ids, one offset, one
//      value or vector) computes the item's byte length;
//   2. an exclusive scan gives every item's byte offset;
//   3. a block formats 128 consecutive items into shared memory at their final
//      relative offsets and copies the block's byte range out with 16-byte
//      stores (items too long for the staging area are written in place).
// The short XML lines between sections are written from the host. The output
// goes to a device buffer, a host buffer, or a file; a file is streamed in
// chunks through two device staging buffers and two pinned host buffers, so
// that formatting and the device-to-host copy of one chunk overlap the fwrite
// of the previous one.
//
// Field order: the reference iterates its HashMap of fields, an order Rust
// leaves unspecified; here scalar fields come first, then vector fields, each
// in the order given (the reference's two loops), which is one of the orders
// the reference can produce.
#include <cub/cub.cuh>

#include <cstdio>
#include <string>
#include <vector>

#include "decimal.cuh"
#include "objects.h"

namespace geo {
namespace {

constexpr int kItemsPerBlock = 128;
constexpr int kStageBytes = 24 * 1024;

// ------------------------------------------------------------------ items
struct PointsItem {  // indent spaces, "x y z\n" (SoA coordinates)
    const double* xyz;
    int64_t n;
    int indent;
    __device__ int len(int64_t i) const {
        return indent + 3 + f64_text(xyz[i]).len + f64_text(xyz[n + i]).len + f64_text(xyz[2 * n + i]).len;
    }
    __device__ void write(int64_t i, char* p) const {
        for (int j = 0; j < indent; ++j) p[j] = ' ';
        p += indent;
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
            const F64Text t = f64_text(xyz[c * n + i]);
            f64_write(t, p);
            p += t.len;
            *p++ = c < 2 ? ' ' : '\n';
        }
    }
};

struct ConnItem {  // "id " for the 10 nodes of an element
    const int32_t* conn;
    int64_t n;
    __device__ int len(int64_t e) const {
        int s = 0;
#pragma unroll
        for (int j = 0; j < 10; ++j) s += uint_len((uint32_t)conn[j * n + e]) + 1;
        return s;
    }
    __device__ void write(int64_t e, char* p) const {
#pragma unroll 1
        for (int j = 0; j < 10; ++j) {
            const uint32_t v = (uint32_t)conn[j * n + e];
            const int l = uint_len(v);
            uint_write(v, l, p);
            p[l] = ' ';
            p += l + 1;
        }
    }
};

struct OffsetsItem {  // "10(e+1) "
    __device__ int len(int64_t e) const { return uint_len(10 * (uint64_t)(e + 1)) + 1; }
    __device__ void write(int64_t e, char* p) const {
        const uint64_t v = 10 * (uint64_t)(e + 1);
        const int l = uint_len(v);
        uint_write(v, l, p);
        p[l] = ' ';
    }
};

struct TypesItem {  // "24 "
    __device__ int len(int64_t) const { return 3; }
    __device__ void write(int64_t, char* p) const {
        p[0] = '2';
        p[1] = '4';
        p[2] = ' ';
    }
};

struct ValuesItem {  // "v " (scalar) or "x y z " (vector): `comps` values per item
    const double* v;
    int comps;
    __device__ int len(int64_t i) const {
        int s = 0;
        for (int c = 0; c < comps; ++c) s += f64_text(v[comps * i + c]).len + 1;
        return s;
    }
    __device__ void write(int64_t i, char* p) const {
#pragma unroll 1
        for (int c = 0; c < comps; ++c) {
            const F64Text t = f64_text(v[comps * i + c]);
            f64_write(t, p);
            p[t.len] = ' ';
            p += t.len + 1;
        }
    }
};

struct LineItem {  // indent spaces, then `comps` values separated by ' ', then '\n' (AoS data)
    const double* v;
    int comps;
    int indent;
    __device__ int len(int64_t i) const {
        int s = indent + comps;
        for (int c = 0; c < comps; ++c) s += f64_text(v[comps * i + c]).len;
        return s;
    }
    __device__ void write(int64_t i, char* p) const {
        for (int j = 0; j < indent; ++j) p[j] = ' ';
        p += indent;
#pragma unroll 1
        for (int c = 0; c < comps; ++c) {
            const F64Text t = f64_text(v[comps * i + c]);
            f64_write(t, p);
            p[t.len] = c + 1 < comps ? ' ' : '\n';
            p += t.len + 1;
        }
    }
};

struct LegacyCellItem {  // "10 id id ... id\n"
    const int32_t* conn;
    int64_t n;
    __device__ int len(int64_t e) const {
        int s = 3;
#pragma unroll
        for (int j = 0; j < 10; ++j) s += uint_len((uint32_t)conn[j * n + e]) + 1;
        return s;
    }
    __device__ void write(int64_t e, char* p) const {
        p[0] = '1';
        p[1] = '0';
        p += 2;
#pragma unroll 1
        for (int j = 0; j < 10; ++j) {
            const uint32_t v = (uint32_t)conn[j * n + e];
            const int l = uint_len(v);
            *p++ = ' ';
            uint_write(v, l, p);
            p += l;
        }
        *p = '\n';
    }
};

struct LegacyTypeItem {  // "24\n"
    __device__ int len(int64_t) const { return 3; }
    __device__ void write(int64_t, char* p) const {
        p[0] = '2';
        p[1] = '4';
        p[2] = '\n';
    }
};

// ------------------------------------------------------------------ kernels
// Cell value -> node: the sum over the node's elements in increasing element order
// (the incidence list is sorted by element), divided by the number of elements when
// `counted` (write_nodal_vtu averages only when its PlasticStrain pass counted).
__global__ void k_cell_to_node(const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                               const double* __restrict__ cell, int64_t N, int counted, double* __restrict__ out) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
        const int b = inc_ptr[n], e = inc_ptr[n + 1];
        double s = 0.0;
        if (cell)
            for (int j = b; j < e; ++j) s += cell[inc[j] / 10];
        if (counted && e > b) s /= (double)(e - b);
        out[n] = s;
    }
}

template <class Item>
__global__ void __launch_bounds__(256) k_item_lengths(Item it, int64_t n, int64_t* __restrict__ len,
                                                      unsigned long long* __restrict__ max_len) {
    unsigned long long m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int l = it.len(i);
        len[i] = l;
        m = m > (unsigned long long)l ? m : (unsigned long long)l;
    }
    m = __reduce_max_sync(0xffffffffu, (unsigned)m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(max_len, m);
}

// Items [a, b) into dst, item i at dst[off[i] - base].
template <class Item>
__global__ void __launch_bounds__(kItemsPerBlock) k_item_write(Item it, int64_t a, int64_t b,
                                                               const int64_t* __restrict__ off, int64_t base,
                                                               char* __restrict__ dst) {
    __shared__ __align__(16) char stage[kStageBytes + 16];
    for (int64_t b0 = a + (int64_t)blockIdx.x * kItemsPerBlock; b0 < b; b0 += (int64_t)gridDim.x * kItemsPerBlock) {
        const int64_t b1 = b0 + kItemsPerBlock < b ? b0 + kItemsPerBlock : b;
        const int64_t g0 = off[b0] - base, span = off[b1] - base - g0;
        const int lead = (int)((uintptr_t)(dst + g0) & 15);
        const bool staged = span + lead <= kStageBytes;
        const int64_t i = b0 + threadIdx.x;
        if (i < b1) {
            const int64_t o = off[i] - base;
            it.write(i, staged ? stage + lead + (o - g0) : dst + o);
        }
        __syncthreads();
        if (staged) {
            char* d = dst + g0;
            const int64_t head = ((16 - lead) & 15) < span ? ((16 - lead) & 15) : span;
            for (int64_t t = threadIdx.x; t < head; t += kItemsPerBlock) d[t] = stage[lead + t];
            const int64_t nvec = (span - head) >> 4;
            const uint4* s4 = reinterpret_cast<const uint4*>(stage + lead + head);
            uint4* d4 = reinterpret_cast<uint4*>(d + head);
            for (int64_t t = threadIdx.x; t < nvec; t += kItemsPerBlock) d4[t] = s4[t];
            for (int64_t t = head + 16 * nvec + threadIdx.x; t < span; t += kItemsPerBlock) d[t] = stage[lead + t];
        }
        __syncthreads();
    }
}

__global__ void k_fill_iota_offsets(int64_t* off, int64_t n, int64_t stride) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
        off[i] = i * stride;
}

// ------------------------------------------------------------------ host side
struct FieldIn {
    std::string name;
    const double* data;  // host or device, as the caller passed it
    int64_t count;
    int comps;
};

enum Mode { SIZE_ONLY, TO_DEVICE, TO_HOST, TO_FILE };

class Emitter {
public:
    Emitter(geo_ctx* ctx, Mode mode, char* out, int64_t cap, FILE* fp)
        : ctx_(ctx), s_(ctx->stream), mode_(mode), out_(out), cap_(cap), fp_(fp) {}
    ~Emitter() {
        for (auto& e : ev_)
            if (e) cudaEventDestroy(e);
    }

    int64_t pos() const { return pos_; }
    // a field's values on the device (host data copied into the context scratch)
    const double* stage(const double* data, size_t n) {
        if (mode_ == TO_FILE) flush_pending();
        return stage_in(ctx_, SCR_IN0, data, n);
    }
    // true when the output did not fit the buffer (the size is still counted)
    bool overflow() const { return overflow_; }

    void text(const std::string& str) {
        reserve((int64_t)str.size());
        if (mode_ == TO_DEVICE) GEO_CUDA(cudaMemcpyAsync(out_ + pos_, str.data(), str.size(), cudaMemcpyHostToDevice, s_));
        if (mode_ == TO_HOST) std::memcpy(out_ + pos_, str.data(), str.size());
        if (mode_ == TO_FILE) {
            flush_pending();
            put(str.data(), str.size());
        }
        pos_ += (int64_t)str.size();
    }

    template <class Item>
    void section(const Item& it, int64_t n, int fixed = 0) {
        if (n <= 0) return;
        // the previous section's chunks must have left the staging buffers first
        if (mode_ == TO_FILE) flush_pending();
        int64_t* off = ctx_scratch<int64_t>(ctx_, SCR_TMP1, (size_t)n + 1);
        const unsigned grid = blocks(n, 256);
        int64_t max_len = fixed;
        if (fixed) {
            k_fill_iota_offsets<<<grid, 256, 0, s_>>>(off, n, fixed);
            check_launch(ctx_, "k_fill_iota_offsets");
        } else {
            int64_t* len = ctx_scratch<int64_t>(ctx_, SCR_TMP0, (size_t)n + 1);
            unsigned long long* umax = ctx_scratch<unsigned long long>(ctx_, SCR_OUT1, 1);
            GEO_CUDA(cudaMemsetAsync(umax, 0, sizeof(unsigned long long), s_));
            GEO_CUDA(cudaMemsetAsync(len + n, 0, sizeof(int64_t), s_));
            k_item_lengths<<<grid, 256, 0, s_>>>(it, n, len, umax);
            check_launch(ctx_, "k_item_lengths");
            size_t tmp_bytes = 0;
            GEO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, len, off, n + 1, s_));
            unsigned char* tmp = ctx_scratch<unsigned char>(ctx_, SCR_TMP2, tmp_bytes);
            GEO_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, len, off, n + 1, s_));
            GEO_CUDA(cudaMemcpyAsync(host_.m, umax, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s_));
        }
        GEO_CUDA(cudaMemcpyAsync(&host_.total, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
        GEO_CUDA(cudaStreamSynchronize(s_));
        if (!fixed) max_len = (int64_t)host_.m[0];
        const int64_t total = host_.total;
        reserve(total);
        if (mode_ == SIZE_ONLY) {
            pos_ += total;
            return;
        }
        if (mode_ == TO_DEVICE) {
            k_item_write<<<blocks(n, kItemsPerBlock), kItemsPerBlock, 0, s_>>>(it, 0, n, off, -pos_, out_);
            check_launch(ctx_, "k_item_write");
            pos_ += total;
            return;
        }
        // chunked through the staging buffers: chunk boundaries every m items
        const int64_t m = std::max<int64_t>(1, kChunkBytes / std::max<int64_t>(1, max_len));
        const int64_t nchunks = cdiv(n, m);
        std::vector<int64_t> bounds((size_t)nchunks + 1);
        GEO_CUDA(cudaMemcpy2DAsync(bounds.data(), sizeof(int64_t), off, (size_t)m * sizeof(int64_t),
                                   sizeof(int64_t), (size_t)nchunks, cudaMemcpyDeviceToHost, s_));
        GEO_CUDA(cudaStreamSynchronize(s_));
        bounds[(size_t)nchunks] = total;
        for (int64_t c = 0; c < nchunks; ++c) {
            const int64_t a = c * m, b = std::min(n, a + m);
            const int64_t bytes = bounds[(size_t)c + 1] - bounds[(size_t)c];
            const int slot = slot_;
            if (mode_ == TO_FILE) wait_slot(slot);
            char* dst = ctx_scratch<char>(ctx_, slot ? SCR_IN1 : SCR_OUT0, stage_size(bytes));
            k_item_write<<<blocks(b - a, kItemsPerBlock), kItemsPerBlock, 0, s_>>>(it, a, b, off,
                                                                                  bounds[(size_t)c], dst);
            check_launch(ctx_, "k_item_write");
            if (mode_ == TO_HOST) {
                GEO_CUDA(cudaMemcpyAsync(out_ + pos_, dst, (size_t)bytes, cudaMemcpyDeviceToHost, s_));
                GEO_CUDA(cudaStreamSynchronize(s_));
            } else {
                ctx_->pinned[slot].ensure(stage_size(bytes));
                GEO_CUDA(cudaMemcpyAsync(ctx_->pinned[slot].p, dst, (size_t)bytes, cudaMemcpyDeviceToHost, s_));
                if (!ev_[slot]) GEO_CUDA(cudaEventCreateWithFlags(&ev_[slot], cudaEventDisableTiming));
                GEO_CUDA(cudaEventRecord(ev_[slot], s_));
                pending_[slot] = bytes;
                order_[slot] = seq_++;
                slot_ ^= 1;
            }
            pos_ += bytes;
        }
    }

    void finish() {
        if (mode_ == TO_FILE) {
            flush_pending();
            if (std::fflush(fp_) != 0) fail(GEO_ERR_INVALID_ARG, "write to the output file failed");
        }
        if (mode_ == TO_DEVICE) GEO_CUDA(cudaStreamSynchronize(s_));
    }

private:
    static constexpr int64_t kChunkBytes = int64_t(64) << 20;

    // a buffer sink that cannot take `bytes` more stops writing and only counts
    void reserve(int64_t bytes) {
        if ((mode_ == TO_DEVICE || mode_ == TO_HOST) && pos_ + bytes > cap_) {
            overflow_ = true;
            mode_ = SIZE_ONLY;
        }
    }

    unsigned blocks(int64_t n, int bs) const {
        const int64_t cap = (int64_t)ctx_->sm_count * 16;
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, bs), cap));
    }
    // staging sizes grow in powers of two from 1 MB, so the context's buffers settle
    static size_t stage_size(int64_t bytes) {
        size_t s = size_t(1) << 20;
        while ((int64_t)s < bytes) s <<= 1;
        return s;
    }
    void put(const char* p, size_t n) {
        if (n && std::fwrite(p, 1, n, fp_) != n) fail(GEO_ERR_INVALID_ARG, "write to the output file failed");
    }
    // writes out the chunk held in a slot (its copy must have completed first)
    void wait_slot(int slot) {
        if (!pending_[slot]) return;
        // the other slot may hold an older chunk: keep file order
        const int other = slot ^ 1;
        if (pending_[other] && order_[other] < order_[slot]) wait_slot(other);
        GEO_CUDA(cudaEventSynchronize(ev_[slot]));
        put(ctx_->pinned[slot].p, (size_t)pending_[slot]);
        pending_[slot] = 0;
    }
    void flush_pending() {
        const int first = (pending_[0] && pending_[1]) ? (order_[0] < order_[1] ? 0 : 1) : (pending_[0] ? 0 : 1);
        wait_slot(first);
        wait_slot(first ^ 1);
    }

    geo_ctx* ctx_;
    cudaStream_t s_;
    Mode mode_;
    char* out_;
    int64_t cap_;
    FILE* fp_;
    int64_t pos_ = 0;
    bool overflow_ = false;
    struct {
        unsigned long long m[1];
        int64_t total;
    } host_{};
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    int64_t pending_[2] = {0, 0};
    int64_t order_[2] = {0, 0};
    int64_t seq_ = 0;
    int slot_ = 0;
};

void emit_fields(Emitter& em, const std::vector<FieldIn>& fields) {
    for (int pass = 0; pass < 2; ++pass)
        for (const FieldIn& f : fields) {
            const bool vec = f.comps == 3;
            if (vec != (pass == 1)) continue;
            em.text("        <DataArray type=\"Float64\" Name=\"" + f.name +
                    (vec ? "\" NumberOfComponents=\"3\" format=\"ascii\">\n" : "\" format=\"ascii\">\n") +
                    "          ");
            em.section(ValuesItem{em.stage(f.data, (size_t)(f.count * f.comps)), f.comps}, f.count);
            em.text("\n        </DataArray>\n");
        }
}

// The XML header, points and cells shared by write_vtu and write_nodal_vtu (vtk_writer.rs:104-174, :536-576)
void emit_vtu_head(Emitter& em, const geo_mesh* m) {
    const int64_t N = m->n_nodes, E = m->n_elem;
    em.text("<?xml version=\"1.0\"?>\n"
            "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n"
            "  <UnstructuredGrid>\n"
            "    <Piece NumberOfPoints=\"" + std::to_string(N) + "\" NumberOfCells=\"" + std::to_string(E) +
            "\">\n"
            "      <Points>\n"
            "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    em.section(PointsItem{m->xyz.p, N, 10}, N);
    em.text("        </DataArray>\n"
            "      </Points>\n"
            "      <Cells>\n"
            "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n"
            "          ");
    em.section(ConnItem{m->conn.p, E}, E);
    em.text("\n        </DataArray>\n"
            "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n"
            "          ");
    em.section(OffsetsItem{}, E);
    em.text("\n        </DataArray>\n"
            "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n"
            "          ");
    em.section(TypesItem{}, E, 3);
    em.text("\n        </DataArray>\n"
            "      </Cells>\n");
}

const char* const kTail = "    </Piece>\n"
                          "  </UnstructuredGrid>\n"
                          "</VTKFile>\n";

// VtkWriter::write_vtu's sequence of writes (vtk_writer.rs:104-265)
void emit_vtu(Emitter& em, const geo_mesh* m, const std::vector<FieldIn>& pf, const std::vector<FieldIn>& cf) {
    emit_vtu_head(em, m);
    if (!pf.empty()) {
        em.text("      <PointData>\n");
        emit_fields(em, pf);
        em.text("      </PointData>\n");
    }
    if (!cf.empty()) {
        em.text("      <CellData>\n");
        emit_fields(em, cf);
        em.text("      </CellData>\n");
    }
    em.text(kTail);
    em.finish();
}

// VtkWriter::write's sequence of writes (vtk_writer.rs:13-101): legacy ASCII .vtk
void emit_vtk_legacy(Emitter& em, const geo_mesh* m, const std::vector<FieldIn>& pf,
                     const std::vector<FieldIn>& cf) {
    const int64_t N = m->n_nodes, E = m->n_elem;
    em.text("# vtk DataFile Version 3.0\n"
            "Tet10 Mesh generated by geo_simulator\n"
            "ASCII\n"
            "DATASET UNSTRUCTURED_GRID\n"
            "POINTS " + std::to_string(N) + " double\n");
    em.section(PointsItem{m->xyz.p, N, 0}, N);
    em.text("\nCELLS " + std::to_string(E) + " " + std::to_string(11 * E) + "\n");
    em.section(LegacyCellItem{m->conn.p, E}, E);
    em.text("\nCELL_TYPES " + std::to_string(E) + "\n");
    em.section(LegacyTypeItem{}, E, 3);
    auto block = [&](const char* tag, int64_t count, const std::vector<FieldIn>& fields) {
        if (fields.empty()) return;
        em.text(std::string("\n") + tag + " " + std::to_string(count) + "\n");
        for (int pass = 0; pass < 2; ++pass)
            for (const FieldIn& f : fields) {
                const bool vec = f.comps == 3;
                if (vec != (pass == 1)) continue;
                em.text(vec ? "VECTORS " + f.name + " double\n"
                            : "SCALARS " + f.name + " double 1\nLOOKUP_TABLE default\n");
                em.section(LineItem{em.stage(f.data, (size_t)(f.count * f.comps)), f.comps, 0}, f.count);
            }
    };
    block("POINT_DATA", N, pf);
    block("CELL_DATA", E, cf);
    em.finish();
}

// the nine cell fields write_nodal_vtu averages to the nodes, in its output order
const char* const kNodalNames[9] = {"PlasticStrain", "Stress_II",   "StrainRate_II",    "Pressure",        "Viscosity",
                                    "IsYielding",    "YieldStress", "PlasticViscosity", "SoftenedCohesion"};

// VtkWriter::write_nodal_vtu's sequence of writes (vtk_writer.rs:531-789)
void emit_vtu_nodal(Emitter& em, geo_mesh* m, const std::vector<FieldIn>& pf, const std::vector<FieldIn>& cf) {
    const int64_t N = m->n_nodes;
    const FieldIn* src[9] = {};
    for (int k = 0; k < 9; ++k)
        for (const FieldIn& f : cf)
            if (f.comps == 1 && f.name == kNodalNames[k]) src[k] = &f;  // the map keeps the last of a name
    for (const FieldIn* f : src)
        if (f) GEO_CHECK_ARG(f->count >= m->n_elem, "nodal VTU: a named cell field has fewer values than cells");
    emit_vtu_head(em, m);
    em.text("      <PointData>\n");
    for (const FieldIn& f : pf) {
        if (f.comps != 3) continue;
        em.text("        <DataArray type=\"Float64\" Name=\"" + f.name +
                "\" NumberOfComponents=\"3\" format=\"ascii\">\n");
        em.section(LineItem{em.stage(f.data, (size_t)(f.count * 3)), 3, 10}, f.count);
        em.text("        </DataArray>\n");
    }
    auto scalar = [&](const std::string& name, const double* v, int64_t n) {
        em.text("        <DataArray type=\"Float64\" Name=\"" + name + "\" format=\"ascii\">\n          ");
        em.section(ValuesItem{v, 1}, n);
        em.text("\n        </DataArray>\n");
    };
    for (const FieldIn& f : pf)
        if (f.comps == 1) scalar(f.name, em.stage(f.data, (size_t)f.count), f.count);
    ensure_inverse_map(m);
    geo_ctx* ctx = m->ctx;
    for (int k = 0; k < 9; ++k) {
        const double* cell = src[k] ? em.stage(src[k]->data, (size_t)m->n_elem) : nullptr;
        double* nodal = ctx_scratch<double>(ctx, SCR_IN2, (size_t)N);
        k_cell_to_node<<<(unsigned)std::min<int64_t>(cdiv(N, 256), (int64_t)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
            m->inc_ptr.p, m->inc.p, cell, N, src[0] != nullptr, nodal);
        check_launch(ctx, "k_cell_to_node");
        scalar(kNodalNames[k], nodal, N);
    }
    em.text("      </PointData>\n");
    em.text(kTail);
    em.finish();
}

void emit_format(Emitter& em, geo_mesh* m, int format, const std::vector<FieldIn>& pf,
                 const std::vector<FieldIn>& cf) {
    if (format == GEO_VTK_LEGACY) emit_vtk_legacy(em, m, pf, cf);
    else if (format == GEO_VTK_XML_NODAL) emit_vtu_nodal(em, m, pf, cf);
    else emit_vtu(em, m, pf, cf);
}

std::vector<FieldIn> check_fields(const geo_vtu_field* f, int32_t n) {
    GEO_CHECK_ARG(n >= 0 && (n == 0 || f), "fields array is NULL");
    std::vector<FieldIn> out;
    for (int32_t i = 0; i < n; ++i) {
        GEO_CHECK_ARG(f[i].name, "field name is NULL");
        GEO_CHECK_ARG(f[i].components == 1 || f[i].components == 3, "field components must be 1 or 3");
        GEO_CHECK_ARG(f[i].count >= 0 && (f[i].count == 0 || f[i].data), "field data is NULL");
        out.push_back(FieldIn{f[i].name, f[i].data, f[i].count, f[i].components});
    }
    return out;
}

}  // namespace
}  // namespace geo

using namespace geo;

extern "C" {

int geo_vtk_render(geo_ctx* ctx, const geo_mesh* mesh, int32_t format, const geo_vtu_field* point_fields,
                   int32_t n_point, const geo_vtu_field* cell_fields, int32_t n_cell, char* out, int64_t capacity,
                   int64_t* size) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && size, "ctx/mesh/size is NULL");
    GEO_CHECK_ARG(format == GEO_VTK_LEGACY || format == GEO_VTK_XML || format == GEO_VTK_XML_NODAL,
                  "unknown VTK format");
    const auto pf = check_fields(point_fields, n_point);
    const auto cf = check_fields(cell_fields, n_cell);
    Emitter em(ctx, out ? (is_device_ptr(out) ? TO_DEVICE : TO_HOST) : SIZE_ONLY, out, out ? capacity : 0, nullptr);
    emit_format(em, const_cast<geo_mesh*>(mesh), format, pf, cf);
    *size = em.pos();
    if (em.overflow()) fail(GEO_ERR_INVALID_ARG, "output buffer too small (size holds the required bytes)");
    GEO_API_END
}

int geo_write_vtk(geo_ctx* ctx, const geo_mesh* mesh, int32_t format, const geo_vtu_field* point_fields,
                  int32_t n_point, const geo_vtu_field* cell_fields, int32_t n_cell, const char* path, int64_t* size) {
    GEO_API_BEGIN(ctx)
    GEO_CHECK_ARG(ctx && mesh && path, "ctx/mesh/path is NULL");
    GEO_CHECK_ARG(format == GEO_VTK_LEGACY || format == GEO_VTK_XML || format == GEO_VTK_XML_NODAL,
                  "unknown VTK format");
    const auto pf = check_fields(point_fields, n_point);
    const auto cf = check_fields(cell_fields, n_cell);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) fail(GEO_ERR_INVALID_ARG, std::string("cannot create ") + path);
    try {
        Emitter em(ctx, TO_FILE, nullptr, 0, fp);
        emit_format(em, const_cast<geo_mesh*>(mesh), format, pf, cf);
        if (size) *size = em.pos();
    } catch (...) {
        std::fclose(fp);
        throw;
    }
    if (std::fclose(fp) != 0) fail(GEO_ERR_INVALID_ARG, "closing the output file failed");
    GEO_API_END
}

int geo_vtu_render(geo_ctx* ctx, const geo_mesh* mesh, const geo_vtu_field* point_fields, int32_t n_point,
                   const geo_vtu_field* cell_fields, int32_t n_cell, char* out, int64_t capacity, int64_t* size) {
    return geo_vtk_render(ctx, mesh, GEO_VTK_XML, point_fields, n_point, cell_fields, n_cell, out, capacity, size);
}

int geo_write_vtu(geo_ctx* ctx, const geo_mesh* mesh, const geo_vtu_field* point_fields, int32_t n_point,
                  const geo_vtu_field* cell_fields, int32_t n_cell, const char* path, int64_t* size) {
    return geo_write_vtk(ctx, mesh, GEO_VTK_XML, point_fields, n_point, cell_fields, n_cell, path, size);
}

}  // extern "C"
