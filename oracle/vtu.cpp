// CPU oracle for the VTU writer -- TEST INFRASTRUCTURE ONLY.
//
// Restates VtkWriter::write_vtu (mesh/vtk_writer.rs:104-265): ASCII XML with
// the points, connectivity, offsets, types and the point / cell fields, every
// f64 printed with Rust's `{}` (core::fmt Display for f64), every index with
// `{}` for usize.
//
// Rust's Display for f64 (core::fmt::float, flt2dec::to_shortest_str with no
// fractional minimum) is restated from its published algorithm:
//  * decoding (flt2dec::decoder): v = c * 2^q; a normal value whose fraction bits
//    are all zero has the asymmetric interval [v - 2^(q-2), v + 2^(q-1)], every
//    other finite value [v - 2^(q-1), v + 2^(q-1)]; the end points belong to the
//    interval iff c is even;
//  * shortest digits (Steele & White free-format / Dragon4, which Grisu defers
//    to when unsure): scanning decimal positions from the one above v's leading
//    digit downwards, stop at the first position 10^e at which the interval
//    holds floor(v / 10^e) * 10^e or the next multiple; emit the one inside, the
//    one nearer v when both are;
//  * layout: value 0.d1..dn * 10^x printed positionally -- "0.00ddd" for x <= 0,
//    "dd.dd" for 0 < x < n, "ddd000" for x >= n -- never with an exponent; "-"
//    for negative values including -0; "NaN", "inf", "-inf".
// Exactness comes from glibc: long double holds v and both interval end points
// exactly, and "%.800Le" prints their exact decimal expansions; candidates are
// short decimal strings; all comparisons are on exact decimal digit strings.
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "oracle.h"

namespace {

// Exact positive decimal: value = 0.digits * 10^exp10, digits[0] != '0'.
struct Dec {
    std::string digits;
    int exp10 = 0;
};

Dec exact_decimal(long double x) {
    char buf[1000];
    std::snprintf(buf, sizeof buf, "%.800Le", x);
    Dec d;
    const char* p = buf;
    for (; *p && *p != 'e'; ++p)
        if (*p >= '0' && *p <= '9') d.digits.push_back(*p);
    const int e = std::atoi(p + 1);
    d.exp10 = e + 1;
    while (d.digits.size() > 1 && d.digits.back() == '0') d.digits.pop_back();
    return d;
}

// -1, 0, +1 for a < b, a == b, a > b (both positive, normalised)
int cmp(const Dec& a, const Dec& b) {
    if (a.exp10 != b.exp10) return a.exp10 < b.exp10 ? -1 : 1;
    const size_t n = std::max(a.digits.size(), b.digits.size());
    for (size_t i = 0; i < n; ++i) {
        const char ca = i < a.digits.size() ? a.digits[i] : '0';
        const char cb = i < b.digits.size() ? b.digits[i] : '0';
        if (ca != cb) return ca < cb ? -1 : 1;
    }
    return 0;
}

// digits (no leading zero) * 10^pos as a normalised Dec
Dec make_dec(std::string digits, int pos) {
    size_t lead = 0;
    while (lead + 1 < digits.size() && digits[lead] == '0') ++lead;
    digits = digits.substr(lead);
    Dec d;
    d.exp10 = (int)digits.size() + pos;
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    d.digits = digits;
    return d;
}

std::string increment(std::string s) {
    int i = (int)s.size() - 1;
    while (i >= 0 && s[i] == '9') s[i--] = '0';
    if (i < 0) return "1" + s;
    ++s[i];
    return s;
}

// shortest digits of a positive finite double in Rust's sense
Dec shortest(double v) {
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    const int be = (int)((bits >> 52) & 0x7ff);
    const uint64_t frac = bits & ((uint64_t(1) << 52) - 1);
    const uint64_t c = be ? (frac | (uint64_t(1) << 52)) : frac;
    const int q = be ? be - 1075 : -1074;
    const bool irregular = be != 0 && frac == 0;
    const bool inclusive = (c & 1) == 0;
    const long double lv = (long double)v;
    const long double lo = lv - std::ldexp((long double)1, irregular ? q - 2 : q - 1);
    const long double hi = lv + std::ldexp((long double)1, q - 1);
    const Dec V = exact_decimal(lv), L = exact_decimal(lo), H = exact_decimal(hi);
    auto inside = [&](const Dec& x) {
        const int a = cmp(x, L), b = cmp(x, H);
        return inclusive ? (a >= 0 && b <= 0) : (a > 0 && b < 0);
    };
    // position above the leading digit: the only candidate is 10^V.exp10
    {
        const Dec one = make_dec("1", V.exp10);
        if (inside(one)) return one;
    }
    for (int n = 1; n <= 40; ++n) {
        std::string f = V.digits.substr(0, std::min<size_t>(n, V.digits.size()));
        while ((int)f.size() < n) f.push_back('0');
        const int pos = V.exp10 - n;
        const Dec down = make_dec(f, pos), up = make_dec(increment(f), pos);
        const bool din = inside(down), uin = inside(up);
        if (!din && !uin) continue;
        if (din && !uin) return down;
        if (uin && !din) return up;
        // both inside: the nearer one; the remainder of v beyond n digits vs one half
        std::string rem = V.digits.size() > (size_t)n ? V.digits.substr(n) : std::string();
        int r;  // sign of rem - 0.5
        if (rem.empty() || rem[0] < '5') r = -1;
        else if (rem[0] > '5') r = 1;
        else r = rem.find_first_not_of('0', 1) == std::string::npos ? 0 : 1;
        if (r < 0) return down;
        if (r > 0) return up;
        return ((f.back() - '0') % 2 == 0) ? down : up;  // exact tie (does not occur for doubles)
    }
    return V;  // not reached
}

void put_f64(std::string& out, double v) {
    if (std::isnan(v)) {
        out += "NaN";
        return;
    }
    if (std::signbit(v)) out.push_back('-');
    const double a = std::fabs(v);
    if (std::isinf(a)) {
        out += "inf";
        return;
    }
    if (a == 0.0) {
        out.push_back('0');
        return;
    }
    const Dec d = shortest(a);
    const int n = (int)d.digits.size(), x = d.exp10;
    if (x <= 0) {
        out += "0.";
        out.append((size_t)(-x), '0');
        out += d.digits;
    } else if (x < n) {
        out += d.digits.substr(0, (size_t)x);
        out.push_back('.');
        out += d.digits.substr((size_t)x);
    } else {
        out += d.digits;
        out.append((size_t)(x - n), '0');
    }
}

void put_int(std::string& out, int64_t v) { out += std::to_string(v); }

void put_fields(std::string& out, int n_fields, const char* const* names, const double* const* data,
                const int64_t* counts, const int32_t* comps) {
    // scalar fields first, then vector fields (two loops in the reference)
    for (int pass = 0; pass < 2; ++pass)
        for (int f = 0; f < n_fields; ++f) {
            const bool vec = comps[f] == 3;
            if (vec != (pass == 1)) continue;
            out += "        <DataArray type=\"Float64\" Name=\"";
            out += names[f];
            out += vec ? "\" NumberOfComponents=\"3\" format=\"ascii\">\n" : "\" format=\"ascii\">\n";
            out += "          ";
            const int64_t n = counts[f] * (vec ? 3 : 1);
            for (int64_t i = 0; i < n; ++i) {
                put_f64(out, data[f][i]);
                out.push_back(' ');
            }
            out += "\n        </DataArray>\n";
        }
}

const char* const kNodalNames[9] = {"PlasticStrain",    "Stress_II",   "StrainRate_II",
                                     "Pressure",         "Viscosity",   "IsYielding",
                                     "YieldStress",      "PlasticViscosity", "SoftenedCohesion"};

}  // namespace

extern "C" {

// VtkWriter::write (mesh/vtk_writer.rs:13-101): legacy ASCII .vtk
int64_t orc_write_vtk(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, int n_point,
                      const char* const* p_names, const double* const* p_data, const int64_t* p_counts,
                      const int32_t* p_comps, int n_cell, const char* const* c_names, const double* const* c_data,
                      const int64_t* c_counts, const int32_t* c_comps, char* out, int64_t cap) {
    std::string s;
    s += "# vtk DataFile Version 3.0\n";
    s += "Tet10 Mesh generated by geo_simulator\n";
    s += "ASCII\n";
    s += "DATASET UNSTRUCTURED_GRID\n";
    s += "POINTS " + std::to_string(n_nodes) + " double\n";
    for (int64_t i = 0; i < n_nodes; ++i) {
        put_f64(s, xyz[3 * i]);
        s.push_back(' ');
        put_f64(s, xyz[3 * i + 1]);
        s.push_back(' ');
        put_f64(s, xyz[3 * i + 2]);
        s.push_back('\n');
    }
    s += "\nCELLS " + std::to_string(n_elem) + " " + std::to_string(11 * n_elem) + "\n";
    for (int64_t e = 0; e < n_elem; ++e) {
        s += "10";
        for (int l = 0; l < 10; ++l) {
            s.push_back(' ');
            put_int(s, conn[10 * e + l]);
        }
        s.push_back('\n');
    }
    s += "\nCELL_TYPES " + std::to_string(n_elem) + "\n";
    for (int64_t e = 0; e < n_elem; ++e) s += "24\n";
    auto block = [&](const char* tag, int64_t count, int nf, const char* const* names, const double* const* data,
                     const int64_t* counts, const int32_t* comps) {
        if (nf <= 0) return;
        s += std::string("\n") + tag + " " + std::to_string(count) + "\n";
        for (int pass = 0; pass < 2; ++pass)
            for (int f = 0; f < nf; ++f) {
                const bool vec = comps[f] == 3;
                if (vec != (pass == 1)) continue;
                if (!vec) {
                    s += std::string("SCALARS ") + names[f] + " double 1\n";
                    s += "LOOKUP_TABLE default\n";
                    for (int64_t i = 0; i < counts[f]; ++i) {
                        put_f64(s, data[f][i]);
                        s.push_back('\n');
                    }
                } else {
                    s += std::string("VECTORS ") + names[f] + " double\n";
                    for (int64_t i = 0; i < counts[f]; ++i) {
                        put_f64(s, data[f][3 * i]);
                        s.push_back(' ');
                        put_f64(s, data[f][3 * i + 1]);
                        s.push_back(' ');
                        put_f64(s, data[f][3 * i + 2]);
                        s.push_back('\n');
                    }
                }
            }
    };
    block("POINT_DATA", n_nodes, n_point, p_names, p_data, p_counts, p_comps);
    block("CELL_DATA", n_elem, n_cell, c_names, c_data, c_counts, c_comps);
    if (out && (int64_t)s.size() <= cap) std::memcpy(out, s.data(), s.size());
    return (int64_t)s.size();
}

// VtkWriter::write_nodal_vtu (mesh/vtk_writer.rs:531-789): points and cells as in
// write_vtu; PointData holds the vector point fields (one vector per line), the
// scalar point fields, then nine named cell fields averaged to the nodes (summed
// per node in element order; divided by the count that only the PlasticStrain
// pass increments; a missing field leaves zeros). No CellData. Cell fields must
// hold at least n_elem values.
int64_t orc_write_vtu_nodal(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, int n_point,
                            const char* const* p_names, const double* const* p_data, const int64_t* p_counts,
                            const int32_t* p_comps, int n_cell, const char* const* c_names,
                            const double* const* c_data, const int64_t* c_counts, const int32_t* c_comps, char* out,
                            int64_t cap) {
    std::string s;
    s += "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
    s += "  <UnstructuredGrid>\n";
    s += "    <Piece NumberOfPoints=\"" + std::to_string(n_nodes) + "\" NumberOfCells=\"" + std::to_string(n_elem) +
         "\">\n";
    s += "      <Points>\n";
    s += "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    for (int64_t i = 0; i < n_nodes; ++i) {
        s += "          ";
        put_f64(s, xyz[3 * i]);
        s.push_back(' ');
        put_f64(s, xyz[3 * i + 1]);
        s.push_back(' ');
        put_f64(s, xyz[3 * i + 2]);
        s.push_back('\n');
    }
    s += "        </DataArray>\n";
    s += "      </Points>\n";
    s += "      <Cells>\n";
    s += "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
    s += "          ";
    for (int64_t i = 0; i < 10 * n_elem; ++i) {
        put_int(s, conn[i]);
        s.push_back(' ');
    }
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
    s += "          ";
    for (int64_t i = 1; i <= n_elem; ++i) {
        put_int(s, 10 * i);
        s.push_back(' ');
    }
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
    s += "          ";
    for (int64_t i = 0; i < n_elem; ++i) s += "24 ";
    s += "\n        </DataArray>\n";
    s += "      </Cells>\n";
    // cell -> node averaging of the nine named fields
    std::vector<std::vector<double>> nodal(9, std::vector<double>((size_t)n_nodes, 0.0));
    std::vector<int64_t> count((size_t)n_nodes, 0);
    for (int k = 0; k < 9; ++k) {
        const double* src = nullptr;
        for (int f = 0; f < n_cell; ++f)
            if (c_comps[f] == 1 && std::strcmp(c_names[f], kNodalNames[k]) == 0) src = c_data[f];
        if (!src) continue;
        for (int64_t e = 0; e < n_elem; ++e)
            for (int l = 0; l < 10; ++l) {
                const int64_t n = conn[10 * e + l];
                nodal[k][(size_t)n] += src[e];
                if (k == 0) ++count[(size_t)n];
            }
    }
    for (int64_t i = 0; i < n_nodes; ++i)
        if (count[(size_t)i] > 0)
            for (int k = 0; k < 9; ++k) nodal[k][(size_t)i] /= (double)count[(size_t)i];
    s += "      <PointData>\n";
    for (int f = 0; f < n_point; ++f) {
        if (p_comps[f] != 3) continue;
        s += std::string("        <DataArray type=\"Float64\" Name=\"") + p_names[f] +
             "\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (int64_t i = 0; i < p_counts[f]; ++i) {
            s += "          ";
            put_f64(s, p_data[f][3 * i]);
            s.push_back(' ');
            put_f64(s, p_data[f][3 * i + 1]);
            s.push_back(' ');
            put_f64(s, p_data[f][3 * i + 2]);
            s.push_back('\n');
        }
        s += "        </DataArray>\n";
    }
    auto scalar_array = [&](const char* name, const double* v, int64_t n) {
        s += std::string("        <DataArray type=\"Float64\" Name=\"") + name + "\" format=\"ascii\">\n";
        s += "          ";
        for (int64_t i = 0; i < n; ++i) {
            put_f64(s, v[i]);
            s.push_back(' ');
        }
        s += "\n        </DataArray>\n";
    };
    for (int f = 0; f < n_point; ++f)
        if (p_comps[f] == 1) scalar_array(p_names[f], p_data[f], p_counts[f]);
    for (int k = 0; k < 9; ++k) scalar_array(kNodalNames[k], nodal[k].data(), n_nodes);
    s += "      </PointData>\n";
    s += "    </Piece>\n";
    s += "  </UnstructuredGrid>\n";
    s += "</VTKFile>\n";
    (void)c_counts;
    if (out && (int64_t)s.size() <= cap) std::memcpy(out, s.data(), s.size());
    return (int64_t)s.size();
}

int orc_format_f64(double v, char* out, int cap) {
    std::string s;
    put_f64(s, v);
    if ((int)s.size() + 1 > cap) return -1;
    std::memcpy(out, s.c_str(), s.size() + 1);
    return (int)s.size();
}

int64_t orc_write_vtu(int64_t n_nodes, const double* xyz, int64_t n_elem, const int64_t* conn, int n_point,
                      const char* const* p_names, const double* const* p_data, const int64_t* p_counts,
                      const int32_t* p_comps, int n_cell, const char* const* c_names, const double* const* c_data,
                      const int64_t* c_counts, const int32_t* c_comps, char* out, int64_t cap) {
    std::string s;
    s += "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
    s += "  <UnstructuredGrid>\n";
    s += "    <Piece NumberOfPoints=\"";
    put_int(s, n_nodes);
    s += "\" NumberOfCells=\"";
    put_int(s, n_elem);
    s += "\">\n";
    s += "      <Points>\n";
    s += "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    for (int64_t i = 0; i < n_nodes; ++i) {
        s += "          ";
        put_f64(s, xyz[3 * i]);
        s.push_back(' ');
        put_f64(s, xyz[3 * i + 1]);
        s.push_back(' ');
        put_f64(s, xyz[3 * i + 2]);
        s.push_back('\n');
    }
    s += "        </DataArray>\n";
    s += "      </Points>\n";
    s += "      <Cells>\n";
    s += "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
    s += "          ";
    for (int64_t i = 0; i < 10 * n_elem; ++i) {
        put_int(s, conn[i]);
        s.push_back(' ');
    }
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
    s += "          ";
    for (int64_t i = 1; i <= n_elem; ++i) {
        put_int(s, 10 * i);
        s.push_back(' ');
    }
    s += "\n        </DataArray>\n";
    s += "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
    s += "          ";
    for (int64_t i = 0; i < n_elem; ++i) s += "24 ";
    s += "\n        </DataArray>\n";
    s += "      </Cells>\n";
    if (n_point > 0) {
        s += "      <PointData>\n";
        put_fields(s, n_point, p_names, p_data, p_counts, p_comps);
        s += "      </PointData>\n";
    }
    if (n_cell > 0) {
        s += "      <CellData>\n";
        put_fields(s, n_cell, c_names, c_data, c_counts, c_comps);
        s += "      </CellData>\n";
    }
    s += "    </Piece>\n";
    s += "  </UnstructuredGrid>\n";
    s += "</VTKFile>\n";
    if (out && (int64_t)s.size() <= cap) std::memcpy(out, s.data(), s.size());
    return (int64_t)s.size();
}

}  // extern "C"
