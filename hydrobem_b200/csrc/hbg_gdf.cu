// hbg_gdf.cu -- the low-order GDF reader (host code; crates/hydrobem/src/gdf.rs:200-535 and the text
// rules of text.rs:205-345): a label line, ULEN GRAV, ISX ISY, NPAN, then NPAN panels of 4 vertices as
// Fortran list-directed numbers.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydrobem_gpu.h"
#include "hbg_internal.h"

namespace hbg {

// Line breaks as Python's str.splitlines (text.rs:209-230): \n, \r\n, \r, \v, \f, \x1c-\x1e, and the UTF-8
// encodings of U+0085, U+2028, U+2029; the length of the break at i, 0 when none.
static size_t gdf_break_at(const std::string& b, size_t i) {
    const unsigned char c = (unsigned char)b[i];
    if (c == '\r') return i + 1 < b.size() && b[i + 1] == '\n' ? 2 : 1;
    if (c == '\n' || c == '\v' || c == '\f' || (c >= 0x1c && c <= 0x1e)) return 1;
    if (c == 0xc2 && i + 1 < b.size() && (unsigned char)b[i + 1] == 0x85) return 2;
    if (c == 0xe2 && i + 2 < b.size() && (unsigned char)b[i + 1] == 0x80 &&
        ((unsigned char)b[i + 2] == 0xa8 || (unsigned char)b[i + 2] == 0xa9))
        return 3;
    return 0;
}

// Whitespace as Python's str.split (ASCII and the UTF-8 encodings of the Unicode spaces): its length at i.
static size_t gdf_space_at(const std::string& b, size_t i) {
    const unsigned char c = (unsigned char)b[i];
    if (c == ' ' || (c >= 0x09 && c <= 0x0d) || (c >= 0x1c && c <= 0x1f)) return 1;
    const auto at = [&](size_t k) { return i + k < b.size() ? (unsigned char)b[i + k] : 0u; };
    if (c == 0xc2 && (at(1) == 0x85 || at(1) == 0xa0)) return 2;
    if (c == 0xe1 && at(1) == 0x9a && at(2) == 0x80) return 3;
    if (c == 0xe2 && at(1) == 0x80 && ((at(2) >= 0x80 && at(2) <= 0x8a) || at(2) == 0xa8 || at(2) == 0xa9 || at(2) == 0xaf))
        return 3;
    if (c == 0xe2 && at(1) == 0x81 && at(2) == 0x9f) return 3;
    if (c == 0xe3 && at(1) == 0x80 && at(2) == 0x80) return 3;
    return 0;
}

static std::vector<std::string> gdf_lines(const std::string& t) {
    std::vector<std::string> out;
    size_t start = 0, i = 0;
    while (i < t.size()) {
        const size_t n = gdf_break_at(t, i);
        if (n == 0) {
            i++;
            continue;
        }
        out.push_back(t.substr(start, i - start));
        i += n;
        start = i;
    }
    if (start < t.size()) out.push_back(t.substr(start));
    return out;
}

// The tokens of a line, commas taken as spaces (text.rs:232-255).
static std::vector<std::string> gdf_tokens(const std::string& line) {
    std::vector<std::string> out;
    size_t start = 0, i = 0;
    while (i < line.size()) {
        const size_t n = line[i] == ',' ? 1 : gdf_space_at(line, i);
        if (n > 0) {
            if (i > start) out.push_back(line.substr(start, i - start));
            i += n;
            start = i;
        } else {
            i++;
        }
    }
    if (line.size() > start) out.push_back(line.substr(start));
    return out;
}

static std::string gdf_strip(const std::string& s) {
    size_t a = 0, e = s.size();
    while (a < e) {
        const size_t n = gdf_space_at(s, a);
        if (n == 0) break;
        a += n;
    }
    size_t end = a, i = a;
    while (i < e) {
        const size_t n = gdf_space_at(s, i);
        if (n > 0) {
            i += n;
        } else {
            i++;
            end = i;
        }
    }
    return s.substr(a, end - a);
}

// A free-format number [+-]?(d+.?d*|.d+)([eEdD][+-]?d+)? (text.rs:287-325).
static bool gdf_is_number(const std::string& t) {
    size_t i = 0;
    if (i < t.size() && (t[i] == '+' || t[i] == '-')) i++;
    size_t id = 0, fd = 0;
    while (i < t.size() && t[i] >= '0' && t[i] <= '9') i++, id++;
    if (i < t.size() && t[i] == '.') {
        i++;
        while (i < t.size() && t[i] >= '0' && t[i] <= '9') i++, fd++;
    }
    if (id == 0 && fd == 0) return false;
    if (i < t.size() && (t[i] == 'e' || t[i] == 'E' || t[i] == 'd' || t[i] == 'D')) {
        i++;
        if (i < t.size() && (t[i] == '+' || t[i] == '-')) i++;
        size_t ed = 0;
        while (i < t.size() && t[i] >= '0' && t[i] <= '9') i++, ed++;
        if (ed == 0) return false;
    }
    return i == t.size();
}

// Its value, D as the exponent letter, correctly rounded and independent of the locale (text.rs:327-331).
static double gdf_parse(const std::string& tok) {
    std::string t = tok;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';
    size_t s = t[0] == '+' ? 1 : 0;  // from_chars takes no '+'
    double v = 0.0;
    std::from_chars(t.data() + s, t.data() + t.size(), v);
    return v;
}

// Python's repr of a str, as the reference's messages quote a line or a token.
static std::string gdf_repr(const std::string& s) {
    const bool dq = s.find('\'') != std::string::npos && s.find('"') == std::string::npos;
    const char q = dq ? '"' : '\'';
    std::string o(1, q);
    for (char c : s) {
        if (c == q || c == '\\') o += '\\';
        o += c;
    }
    return o + q;
}

static std::string gdf_num(double v) {
    char b[64];
    snprintf(b, sizeof b, "%.17g", v);
    return b;
}

static void gdf_fail(int code, const std::string& msg) { throw Failure{code, msg}; }

// The first n numbers of a line (a comment may follow them).
static std::vector<double> gdf_leading(const std::string& line, size_t n, const char* what, const std::string& path) {
    std::vector<double> v;
    for (const std::string& t : gdf_tokens(line)) {
        if (v.size() == n || !gdf_is_number(t)) break;
        v.push_back(gdf_parse(t));
    }
    if (v.size() < n) gdf_fail(HB_ERR_VALUE, path + ": expected " + what + " on the line " + gdf_repr(gdf_strip(line)));
    return v;
}

static int gdf_integer(double v, const char* name, const std::string& path) {
    if (!(std::isfinite(v) && v == std::floor(v) && std::fabs(v) < 2147483647.0))
        gdf_fail(HB_ERR_VALUE, path + ": " + name + " must be an integer, got " + gdf_num(v));
    return (int)v;
}

static int gdf_flag(double v, const char* name, const std::string& path) {
    const int f = gdf_integer(v, name, path);
    if (f != 0 && f != 1) gdf_fail(HB_ERR_VALUE, path + ": " + name + " must be 0 or 1, not " + std::to_string(f));
    return f;
}

// gdf.rs:511-535 read_low_order_gdf
static void read_gdf(const std::string& path, bool zero_trailer, std::string& label, double& ulen, double& grav,
                     int& isx, int& isy, std::vector<double>& verts) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) gdf_fail(HB_ERR_IO, path + ": " + strerror(errno));
    std::string text;
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    fclose(f);
    const std::vector<std::string> lines = gdf_lines(text);
    if (lines.size() < 4) gdf_fail(HB_ERR_VALUE, path + ": a GDF file needs a header, ULEN GRAV, ISX ISY and NPAN lines");
    label = gdf_strip(lines[0]);
    const std::vector<double> ug = gdf_leading(lines[1], 2, "ULEN GRAV", path);
    ulen = ug[0];
    grav = ug[1];
    if (!(std::isfinite(grav) && grav > 0.0)) gdf_fail(HB_ERR_VALUE, path + ": GRAV must be a positive finite number");
    const std::vector<double> sy = gdf_leading(lines[2], 2, "ISX ISY", path);
    isx = gdf_flag(sy[0], "ISX", path);
    isy = gdf_flag(sy[1], "ISY", path);
    const int npan = gdf_integer(gdf_leading(lines[3], 1, "NPAN", path)[0], "NPAN", path);
    // all remaining numbers: text after a line's numbers is a comment, a line that begins with text is refused
    std::vector<double> values;
    for (size_t l = 4; l < lines.size(); l++) {
        const std::vector<std::string> toks = gdf_tokens(lines[l]);
        for (size_t k = 0; k < toks.size(); k++) {
            if (!gdf_is_number(toks[k])) {
                if (k > 0) break;
                gdf_fail(HB_ERR_VALUE, path + ": line " + std::to_string(l + 1) + ": invalid number " + gdf_repr(toks[k]));
            }
            values.push_back(gdf_parse(toks[k]));
        }
    }
    if (npan < 1) gdf_fail(HB_ERR_VALUE, path + ": NPAN must be >= 1");
    const size_t need = 12 * (size_t)npan;
    if (values.size() < need)
        gdf_fail(HB_ERR_VALUE, path + ": the file ends after " + std::to_string(values.size() / 12) + " of NPAN = " +
                                   std::to_string(npan) + " records");
    if (values.size() > need) {
        bool zeros = true;
        for (size_t i = need; i < values.size(); i++) zeros = zeros && values[i] == 0.0;
        if (!zeros) gdf_fail(HB_ERR_VALUE, path + ": unexpected data after NPAN = " + std::to_string(npan));
        if (!zero_trailer)
            gdf_fail(HB_ERR_VALUE, path + ": trailing record of zeros after NPAN = " + std::to_string(npan) +
                                       " (pass zero_trailer = true)");
    }
    values.resize(need);
    verts.swap(values);
}

}  // namespace hbg

using namespace hbg;

extern "C" HbStatus hbg_read_gdf(const char* path, int32_t zero_trailer, HbgGdf* out) {
    try {
        if (!path || !out) return fail({HB_ERR_ARGUMENT, "null argument"});
        std::string label;
        double ulen = 0.0, grav = 0.0;
        int isx = 0, isy = 0;
        std::vector<double> v;
        read_gdf(path, zero_trailer != 0, label, ulen, grav, isx, isy, v);
        double* p = static_cast<double*>(malloc(sizeof(double) * v.size()));
        if (!p) return fail({HB_ERR_INTERNAL, "out of host memory"});
        memcpy(p, v.data(), sizeof(double) * v.size());
        memset(out->label, 0, sizeof out->label);
        strncpy(out->label, label.c_str(), sizeof out->label - 1);
        out->ulen = ulen;
        out->gravity = grav;
        out->isx = isx;
        out->isy = isy;
        out->n_panels = (int64_t)(v.size() / 12);
        out->vertices = p;
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    } catch (...) {
        return fail({HB_ERR_INTERNAL, "internal error"});
    }
}

extern "C" HbStatus hbg_gdf_free(HbgGdf* g) {
    if (!g) return fail({HB_ERR_ARGUMENT, "null argument"});
    free(g->vertices);
    g->vertices = nullptr;
    g->n_panels = 0;
    return HB_OK;
}
