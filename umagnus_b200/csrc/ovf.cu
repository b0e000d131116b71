// ovf.cu -- field files: OOMMF OVF 1.0 / 2.0 and the legacy dump format.
//
// Host-side restatement of the reference's readers and writers
// (oommf/oommf.go, oommf/ovf1.go, oommf/ovf2.go, oommf/util.go,
// dump/read.go, dump/write.go).  Arrays are host float32, structure of
// arrays [c][z][y][x] (x fastest), the layout of data.Slice.Tensors().
// Numbers in headers and text data are written the way Go's fmt %v writes
// them (shortest round-trip digits, exponent form when the decimal exponent
// is < -4 or >= 6), so files match the reference's byte for byte.
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"


namespace umag {

// ---------------------------------------------------------------- number format
// Go: strconv.FormatFloat(v, 'g', -1, bits) as fmt's %v uses it.
static std::string go_float(double v, int bits) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "+Inf" : "-Inf";
    if (v == 0) return std::signbit(v) ? "-0" : "0";
    char buf[64];
    std::to_chars_result r = bits == 32 ? std::to_chars(buf, buf + sizeof(buf), (float)v, std::chars_format::scientific)
                                        : std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific);
    std::string s(buf, r.ptr);
    // s = [-]d[.ddd]e[+-]XX
    bool neg = s[0] == '-';
    if (neg) s = s.substr(1);
    const size_t e = s.find('e');
    std::string mant = s.substr(0, e);
    const int exp = std::stoi(s.substr(e + 1));
    std::string digits;
    for (char c : mant)
        if (c != '.') digits += c;
    std::string out;
    if (exp < -4 || exp >= 6) {  // %e with the shortest digits
        out = digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        char eb[16];
        snprintf(eb, sizeof(eb), "e%c%02d", exp < 0 ? '-' : '+', exp < 0 ? -exp : exp);
        out += eb;
    } else if (exp >= 0) {  // %f, no trailing zeros
        if ((int)digits.size() <= exp + 1) {
            out = digits + std::string(exp + 1 - digits.size(), '0');
        } else {
            out = digits.substr(0, exp + 1) + "." + digits.substr(exp + 1);
        }
    } else {
        out = "0." + std::string(-exp - 1, '0') + digits;
    }
    return neg ? "-" + out : out;
}

// ---------------------------------------------------------------- helpers
struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(fopen(path, mode)) {}
    ~File() {
        if (f) fclose(f);
    }
};

static size_t nelem(const umag_field_info& in) {
    return (size_t)in.ncomp * in.N[0] * in.N[1] * in.N[2];
}
static void set_str(char* dst, size_t cap, const std::string& s) {
    snprintf(dst, cap, "%s", s.c_str());
}
static std::string trim(const std::string& s, const char* set) {
    size_t a = s.find_first_not_of(set);
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(set);
    return s.substr(a, b - a + 1);
}
static std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// ---------------------------------------------------------------- OVF write
// "# key: " + values joined like fmt.Fprintln (spaces between operands)
static void hdr(std::string& o, const std::string& key, const std::string& val) {
    o += "# " + key + ": " + val + "\n";
}
static std::string f64(double v) { return go_float(v, 64); }

static void write_text_data(std::string& o, const float* src, const umag_field_info& in) {
    const size_t n = (size_t)in.N[0] * in.N[1] * in.N[2];
    for (size_t i = 0; i < n; i++) {  // [z][y][x] cell order, components interleaved
        for (int c = 0; c < in.ncomp; c++) o += go_float(src[c * n + i], 32) + " ";
        o += "\n";
    }
}
static void put_f32(std::string& o, float v, bool big) {
    unsigned char b[4];
    memcpy(b, &v, 4);
    if (big) std::swap(b[0], b[3]), std::swap(b[1], b[2]);
    o.append(reinterpret_cast<char*>(b), 4);
}
static void write_bin4(std::string& o, const float* src, const umag_field_info& in, bool big) {
    put_f32(o, 1234567.0f, big);  // OVF_CONTROL_NUMBER_4
    const size_t n = (size_t)in.N[0] * in.N[1] * in.N[2];
    for (size_t i = 0; i < n; i++)
        for (int c = 0; c < in.ncomp; c++) put_f32(o, src[c * n + i], big);
}

// oommf/ovf2.go:13-81 WriteOVF2, oommf/ovf1.go:14-76 WriteOVF1
static int ovf_write(const char* path, const float* src, const umag_field_info& in, const char* format,
                     int version) {
    const std::string fmt = lower(format ? format : "binary 4");
    const bool text = fmt == "text";
    if (!text && fmt != "binary" && fmt != "binary 4")
        return set_error(UMAG_E_ARG, "illegal OVF data format %s (Text or Binary 4)", format);
    if (version == 1 && in.ncomp != 3) return set_error(UMAG_E_ARG, "OVF1 stores 3-component fields only");
    const double* c = in.cell;
    const int* N = in.N;
    const std::string name = in.title, unit0 = in.unit;
    std::string o;
    if (version == 2) {
        o += "# OOMMF OVF 2.0\n";
        hdr(o, "Segment count", "1");
        hdr(o, "Begin", "Segment");
        hdr(o, "Begin", "Header");
        hdr(o, "Title", name);
        hdr(o, "meshtype", "rectangular");
        hdr(o, "meshunit", "m");
        hdr(o, "xmin", "0");
        hdr(o, "ymin", "0");
        hdr(o, "zmin", "0");
        hdr(o, "xmax", f64(c[0] * N[0]));
        hdr(o, "ymax", f64(c[1] * N[1]));
        hdr(o, "zmax", f64(c[2] * N[2]));
        hdr(o, "valuedim", std::to_string(in.ncomp));
        std::string labels, units;
        const std::string unit = unit0.empty() ? "1" : unit0;
        if (in.ncomp == 1) {
            labels = name;
            units = unit;
        } else {
            for (int i = 0; i < in.ncomp; i++) labels += (i ? " " : "") + name + "_" + std::string(1, (char)('x' + i));
            units = unit + " " + unit + " " + unit;
        }
        hdr(o, "valuelabels", labels);
        hdr(o, "valueunits", units);
        hdr(o, "Desc", "Total simulation time:  " + f64(in.time) + "  s");
        hdr(o, "xbase", f64(c[0] / 2));
        hdr(o, "ybase", f64(c[1] / 2));
        hdr(o, "zbase", f64(c[2] / 2));
        hdr(o, "xnodes", std::to_string(N[0]));
        hdr(o, "ynodes", std::to_string(N[1]));
        hdr(o, "znodes", std::to_string(N[2]));
        hdr(o, "xstepsize", f64(c[0]));
        hdr(o, "ystepsize", f64(c[1]));
        hdr(o, "zstepsize", f64(c[2]));
        hdr(o, "End", "Header");
    } else if (version == 1) {
        hdr(o, "OOMMF", "rectangular mesh v1.0");
        hdr(o, "Segment count", "1");
        hdr(o, "Begin", "Segment");
        hdr(o, "Begin", "Header");
        hdr(o, "Desc", "Time (s) :  " + f64(in.time));
        hdr(o, "Title", name);
        hdr(o, "meshtype", "rectangular");
        hdr(o, "meshunit", "m");
        hdr(o, "xbase", f64(c[0] / 2));
        hdr(o, "ybase", f64(c[1] / 2));
        hdr(o, "zbase", f64(c[2] / 2));
        hdr(o, "xstepsize", f64(c[0]));
        hdr(o, "ystepsize", f64(c[1]));
        hdr(o, "zstepsize", f64(c[2]));
        hdr(o, "xmin", "0");
        hdr(o, "ymin", "0");
        hdr(o, "zmin", "0");
        hdr(o, "xmax", f64(c[0] * N[0]));
        hdr(o, "ymax", f64(c[1] * N[1]));
        hdr(o, "zmax", f64(c[2] * N[2]));
        hdr(o, "xnodes", std::to_string(N[0]));
        hdr(o, "ynodes", std::to_string(N[1]));
        hdr(o, "znodes", std::to_string(N[2]));
        hdr(o, "ValueRangeMinMag", "1e-08");
        hdr(o, "ValueRangeMaxMag", "1");
        hdr(o, "valueunit", unit0);
        hdr(o, "valuemultiplier", "1");
        hdr(o, "End", "Header");
    } else {
        return set_error(UMAG_E_ARG, "OVF version must be 1 or 2");
    }
    const std::string canon = text ? "Text" : "Binary 4";
    hdr(o, "Begin", "Data " + canon);
    if (text) write_text_data(o, src, in);
    else write_bin4(o, src, in, version == 1);  // OVF1 binary is big-endian, OVF2 little-endian
    hdr(o, "End", "Data " + canon);
    hdr(o, "End", "Segment");
    File f(path, "wb");
    if (!f.f) return set_error(UMAG_E_ARG, "cannot create %s", path);
    if (fwrite(o.data(), 1, o.size(), f.f) != o.size()) return set_error(UMAG_E_ARG, "short write to %s", path);
    return UMAG_OK;
}

// ---------------------------------------------------------------- dump
// dump/write.go, dump/read.go: "#dump002", little-endian uint64/float64
// header, float32 data [c][z][y][x], CRC-64 (ISO polynomial) of the frame
static uint64_t crc64_iso(const unsigned char* p, size_t n) {
    static uint64_t tab[256];
    static bool init = false;
    if (!init) {
        for (int i = 0; i < 256; i++) {
            uint64_t c = (uint64_t)i;
            for (int j = 0; j < 8; j++) c = (c & 1) ? (c >> 1) ^ 0xD800000000000000ULL : c >> 1;
            tab[i] = c;
        }
        init = true;
    }
    uint64_t crc = ~0ULL;
    for (size_t i = 0; i < n; i++) crc = tab[(uint8_t)crc ^ p[i]] ^ (crc >> 8);
    return ~crc;
}
static void put_u64(std::string& o, uint64_t v) { o.append(reinterpret_cast<char*>(&v), 8); }
static void put_d(std::string& o, double v) { o.append(reinterpret_cast<char*>(&v), 8); }
static void put_s8(std::string& o, const std::string& s) {
    char b[8] = {};
    memcpy(b, s.data(), s.size() < 8 ? s.size() : 8);
    o.append(b, 8);
}

static int dump_write(const char* path, const float* src, const umag_field_info& in) {
    std::string o;
    put_s8(o, "#dump002");
    put_u64(o, (uint64_t)in.ncomp);
    put_u64(o, (uint64_t)in.N[2]);  // backwards compatible coordinates (z, y, x)
    put_u64(o, (uint64_t)in.N[1]);
    put_u64(o, (uint64_t)in.N[0]);
    put_d(o, in.cell[2]);
    put_d(o, in.cell[1]);
    put_d(o, in.cell[0]);
    put_s8(o, "m");  // mesh unit
    put_d(o, in.time);
    put_s8(o, "s");
    put_s8(o, in.title);
    put_s8(o, in.unit);
    put_u64(o, 4);
    o.append(reinterpret_cast<const char*>(src), sizeof(float) * nelem(in));
    put_u64(o, crc64_iso(reinterpret_cast<const unsigned char*>(o.data()), o.size()));
    File f(path, "wb");
    if (!f.f) return set_error(UMAG_E_ARG, "cannot create %s", path);
    if (fwrite(o.data(), 1, o.size(), f.f) != o.size()) return set_error(UMAG_E_ARG, "short write to %s", path);
    return UMAG_OK;
}

static int slurp(const char* path, std::string* out) {
    File f(path, "rb");
    if (!f.f) return set_error(UMAG_E_ARG, "cannot open %s", path);
    char buf[1 << 16];
    size_t k;
    out->clear();
    while ((k = fread(buf, 1, sizeof(buf), f.f)) > 0) out->append(buf, k);
    return UMAG_OK;
}

static int dump_parse(const std::string& b, umag_field_info* in, float* dst, size_t cap) {
    const size_t hdr_bytes = 8 * 14;
    if (b.size() < hdr_bytes) return set_error(UMAG_E_ARG, "dump: truncated header");
    auto u64 = [&](size_t off) { uint64_t v; memcpy(&v, b.data() + off, 8); return v; };
    auto d64 = [&](size_t off) { double v; memcpy(&v, b.data() + off, 8); return v; };
    auto s8 = [&](size_t off) { std::string s(b.data() + off, 8); return s.substr(0, s.find('\0')); };
    if (s8(0) != "#dump002") return set_error(UMAG_E_ARG, "dump: bad magic number");
    umag_field_info r{};
    r.ncomp = (int)u64(8);
    r.N[2] = (int)u64(16); r.N[1] = (int)u64(24); r.N[0] = (int)u64(32);
    r.cell[2] = d64(40); r.cell[1] = d64(48); r.cell[0] = d64(56);
    r.time = d64(72);
    set_str(r.title, sizeof(r.title), s8(88));
    set_str(r.unit, sizeof(r.unit), s8(96));
    if (u64(104) != 4) return set_error(UMAG_E_ARG, "dump: only single precision supported");
    const size_t n = nelem(r);
    if (b.size() < hdr_bytes + 4 * n + 8) return set_error(UMAG_E_ARG, "dump: truncated data");
    const uint64_t stored = u64(hdr_bytes + 4 * n);
    const uint64_t mine = crc64_iso(reinterpret_cast<const unsigned char*>(b.data()), hdr_bytes + 4 * n);
    if (stored != 0 && stored != mine) return set_error(UMAG_E_ARG, "dump CRC error");
    *in = r;
    if (dst) {
        if (cap < n) return set_error(UMAG_E_ARG, "destination holds %zu floats, the file has %zu", cap, n);
        memcpy(dst, b.data() + hdr_bytes, 4 * n);
    }
    return UMAG_OK;
}

// ---------------------------------------------------------------- OVF read
// oommf/oommf.go:16-46 Read, :85-170 readHeader
static int ovf_parse(const std::string& b, umag_field_info* info, float* dst, size_t cap) {
    size_t pos = 0;
    auto line = [&](std::string* l) -> bool {
        if (pos >= b.size()) return false;
        size_t e = b.find('\n', pos);
        if (e == std::string::npos) e = b.size();
        *l = b.substr(pos, e - pos);
        pos = e + 1;
        return true;
    };
    auto split = [](const std::string& s, std::string* k, std::string* v) {
        size_t c = s.find(':');
        *k = trim(s.substr(0, c), "# ");
        *v = c == std::string::npos ? "" : trim(s.substr(c + 1), "# ");
    };
    std::string l, k, v;
    if (!line(&l)) return set_error(UMAG_E_ARG, "empty field file");
    umag_field_info r{};
    int ovf = 0;
    const std::string first = lower(trim(l, "\r"));
    if (first == "# oommf ovf 2.0") ovf = 2;
    else if (first == "# oommf: rectangular mesh v1.0") { ovf = 1; r.ncomp = 3; }
    else return set_error(UMAG_E_ARG, "unknown header: %s", l.c_str());
    double total_time = 0;
    bool have_t1 = false, have_t2 = false;
    double t1 = 0, t2 = 0;
    std::string format;
    for (;;) {
        if (!line(&l)) return set_error(UMAG_E_ARG, "OVF: no data section");
        l = trim(l, "\r");
        std::string flat = lower(trim(l, "# "));
        std::string nospace;
        for (char ch : flat)
            if (ch != ' ') nospace += ch;
        if (nospace.rfind("begin:data", 0) == 0) {
            split(l, &k, &v);
            std::string val = trim(v, " ");
            // "Data Text" / "Data Binary 4"
            std::string w1, w2, w3;
            size_t a = val.find(' ');
            w1 = val.substr(0, a);
            std::string rest = a == std::string::npos ? "" : trim(val.substr(a + 1), " ");
            size_t c2 = rest.find(' ');
            w2 = rest.substr(0, c2);
            w3 = c2 == std::string::npos ? "" : trim(rest.substr(c2 + 1), " ");
            if (lower(w1) != "data") return set_error(UMAG_E_ARG, "Expected: Begin: Data");
            format = w3.empty() ? "text" : "binary " + w3;
            break;
        }
        split(l, &k, &v);
        const std::string key = lower(k);
        if (key == "title") set_str(r.title, sizeof(r.title), v);
        else if (key == "valueunits") set_str(r.unit, sizeof(r.unit), v.substr(0, v.find(' ')));
        else if (key == "valuedim") r.ncomp = atoi(v.c_str());
        else if (key == "xnodes") r.N[0] = atoi(v.c_str());
        else if (key == "ynodes") r.N[1] = atoi(v.c_str());
        else if (key == "znodes") r.N[2] = atoi(v.c_str());
        else if (key == "xstepsize") r.cell[0] = atof(v.c_str());
        else if (key == "ystepsize") r.cell[1] = atof(v.c_str());
        else if (key == "zstepsize") r.cell[2] = atof(v.c_str());
        else if (key == "desc") {
            size_t c = v.find(':');
            std::string dk = trim(v.substr(0, c), "# ");
            std::string dv = c == std::string::npos ? "" : trim(v.substr(c + 1), "# ");
            if (dk == "Time (s)") { have_t1 = true; t1 = atof(dv.c_str()); }
            if (dk == "Total simulation time") { have_t2 = true; t2 = atof(dv.c_str()); }
        }  // other keys (valuemultiplier, valueunit, bases, ranges) are ignored, as oommf.go:95-128 does
    }
    if (have_t1) total_time = t1;
    if (have_t2) total_time = t2;
    r.time = total_time;
    if (r.cell[0] == 0 && r.cell[1] == 0 && r.cell[2] == 0) r.cell[0] = r.cell[1] = r.cell[2] = 1;
    if (r.ncomp <= 0 || r.N[0] <= 0 || r.N[1] <= 0 || r.N[2] <= 0) return set_error(UMAG_E_ARG, "OVF: bad sizes");
    *info = r;
    if (!dst) return UMAG_OK;
    const size_t n = (size_t)r.N[0] * r.N[1] * r.N[2];
    if (cap < n * r.ncomp) return set_error(UMAG_E_ARG, "destination holds %zu floats, the file has %zu", cap, n * r.ncomp);
    if (format == "text") {
        const char* p = b.c_str() + pos;
        for (size_t i = 0; i < n; i++)
            for (int c = 0; c < r.ncomp; c++) {
                char* end = nullptr;
                const float val = strtof(p, &end);
                if (end == p) return set_error(UMAG_E_ARG, "OVF text: bad number");
                dst[c * n + i] = val;
                p = end;
            }
        return UMAG_OK;
    }
    const bool b8 = format == "binary 8";
    if (!b8 && format != "binary 4") return set_error(UMAG_E_ARG, "unknown format: OVF%d %s", ovf, format.c_str());
    const size_t w = b8 ? 8 : 4;
    if (b.size() < pos + w * (1 + n * r.ncomp)) return set_error(UMAG_E_ARG, "OVF: truncated data");
    const bool big = ovf == 1;  // OVF 1.0 is network byte order
    auto rd = [&](size_t idx) -> double {
        unsigned char x[8];
        memcpy(x, b.data() + pos + idx * w, w);
        if (big)
            for (size_t i = 0; i < w / 2; i++) std::swap(x[i], x[w - 1 - i]);
        if (b8) { double d; memcpy(&d, x, 8); return d; }
        float f; memcpy(&f, x, 4); return f;
    };
    const double ctl = rd(0);
    if (ctl != (b8 ? 123456789012345.0 : 1234567.0))
        return set_error(UMAG_E_ARG, "invalid OVF%d control number: %g", ovf, ctl);
    for (size_t i = 0; i < n; i++)
        for (int c = 0; c < r.ncomp; c++) dst[c * n + i] = (float)rd(1 + i * r.ncomp + c);
    return UMAG_OK;
}

static int field_parse(const std::string& b, umag_field_info* info, float* dst, size_t cap) {
    if (b.compare(0, 8, "#dump002") == 0) return dump_parse(b, info, dst, cap);
    return ovf_parse(b, info, dst, cap);
}

}  // namespace umag

using namespace umag;

extern "C" {
int umag_field_read_info(const char* path, umag_field_info* info) {
    UMAG_REQUIRE(path && info, "NULL argument");
    std::string b;
    UMAG_TRY(slurp(path, &b));
    return field_parse(b, info, nullptr, 0);
}
int umag_field_read(const char* path, float* dst, size_t capacity, umag_field_info* info) {
    UMAG_REQUIRE(path && dst && info, "NULL argument");
    std::string b;
    UMAG_TRY(slurp(path, &b));
    return field_parse(b, info, dst, capacity);
}
int umag_ovf_write(const char* path, const float* src, const umag_field_info* info, const char* format, int version) {
    UMAG_REQUIRE(path && src && info, "NULL argument");
    UMAG_REQUIRE(info->ncomp > 0 && info->N[0] > 0 && info->N[1] > 0 && info->N[2] > 0, "bad field size");
    return ovf_write(path, src, *info, format, version);
}
int umag_dump_write(const char* path, const float* src, const umag_field_info* info) {
    UMAG_REQUIRE(path && src && info, "NULL argument");
    UMAG_REQUIRE(info->ncomp > 0 && info->N[0] > 0 && info->N[1] > 0 && info->N[2] > 0, "bad field size");
    return dump_write(path, src, *info);
}
int umag_format_float(double v, int bits, char* buf, int cap) {
    UMAG_REQUIRE(buf && cap > 0, "NULL argument");
    const std::string s = go_float(v, bits == 32 ? 32 : 64);
    if ((int)s.size() >= cap) return set_error(UMAG_E_ARG, "buffer too small");
    memcpy(buf, s.c_str(), s.size() + 1);
    return UMAG_OK;
}
}
